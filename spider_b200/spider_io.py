"""SPIDER image, stack and document files.

Layout (SPIDER's image_doc and docfile formats):

* A file is unformatted direct-access records of NX 4-byte floats.  The
  header occupies LABREC = ceil(1024 / (4*NX)) records (LABBYT bytes); the
  header words used here (1-based) are NZ(1), NY(2), IREC(3), IFORM(5),
  IMAMI(6), FMAX(7), FMIN(8), AV(9), SIG(10), NX(12), LABREC(13), LABBYT(22),
  LENBYT(23), ISTACK(24), MAXIM(26), IMGNUM(27) and the projection angles
  PSI3/THETA3/PHI3/LANGLE at 101-104 (written by PJ 3Q, writpro_n.f:244-249).
* A simple image/volume is the header followed by NY*NZ records.  A stack is
  an overall header (ISTACK > 0, MAXIM = highest image number) followed, for
  each image, by its own header (IMGNUM) and its data.  An indexed stack has
  ISTACK = -MAXINDX and, after the overall header, INDXREC = ceil(MAXINDX/NX)
  records of raw int32 entries: entry k is the 1-based storage slot of image
  number k (0 = absent), and slot s starts at record
  LABREC + INDXREC + (s-1)*(LABREC + NY*NZ) (lunsethdr.f:215-240,505-530,
  2140-2200).
* Files are native little-endian float32; byte-swapped files are recognised
  by the plausibility of their header words.
* Document files: lines ``key nregs v1 v2 ...``; a ';' in column 2 marks a
  comment.  Angle documents hold psi, theta, phi in registers 1-3 and, for
  RB 3F / RB 32F, the in-plane angle and shifts in registers 6-8.
"""
from __future__ import annotations

import datetime
import math
import os
import re

import numpy as np


# ----------------------------------------------------------------- headers
def _labrec(nx: int) -> int:
    lenbyt = nx * 4
    labrec = 1024 // lenbyt
    if 1024 % lenbyt != 0:
        labrec += 1
    return labrec


def _make_header(nx, ny, nz, iform, *, istack=0, maxim=0, imgnum=0, data=None, angles=None):
    lenbyt = nx * 4
    labrec = _labrec(nx)
    labbyt = labrec * lenbyt
    h = np.zeros(labbyt // 4, np.float32)
    h[0] = nz
    h[1] = ny
    h[2] = labrec + ny * nz if istack == 0 else ny * nz + labrec
    h[4] = iform
    if data is not None:
        d = np.asarray(data, np.float64)
        h[5] = 1
        h[6] = d.max()
        h[7] = d.min()
        h[8] = d.mean()
        h[9] = d.std()
    h[11] = nx
    h[12] = labrec
    h[21] = labbyt
    h[22] = lenbyt
    h[23] = istack
    h[25] = maxim
    h[26] = imgnum
    if angles is not None:
        h[100] = angles[0]   # PSI3
        h[101] = angles[1]   # THETA3
        h[102] = angles[2]   # PHI3
        h[103] = 1.0         # LANGLE
    now = datetime.datetime.now()
    date = now.strftime("%d-%b-%Y").upper().encode()[:11].ljust(12)
    tim = now.strftime("%H:%M:%S").encode()[:8]
    raw = bytearray(h.tobytes())
    raw[211 * 4:211 * 4 + 12] = date
    raw[214 * 4:214 * 4 + 8] = tim
    return np.frombuffer(bytes(raw), np.float32).copy()


def _plausible(h) -> bool:
    try:
        nz, ny, iform, nx, labrec = float(h[0]), float(h[1]), float(h[4]), float(h[11]), float(h[12])
    except Exception:
        return False
    if not all(math.isfinite(v) for v in (nz, ny, iform, nx, labrec)):
        return False
    return (1 <= nx <= 1 << 20 and 1 <= ny <= 1 << 20 and -1 <= nz <= 1 << 20 and
            int(iform) in (1, 3, -11, -12, -21, -22, 0) and labrec >= 1)


def read_header(path):
    """Returns (header float32 array, byte order '<' or '>')."""
    with open(path, "rb") as f:
        raw = f.read(1024)
    if len(raw) < 256 * 4 // 4 * 4:
        raise ValueError(f"{path}: too short for a SPIDER header")
    for order in ("<", ">"):
        h = np.frombuffer(raw[:1024], dtype=order + "f4")
        if _plausible(h):
            return h.astype(np.float32), order
    raise ValueError(f"{path}: not a SPIDER image (implausible header)")


def _geom(h):
    nz = max(int(h[0]), 1)
    return int(h[11]), int(h[1]), nz, int(h[21])


def read_image(path):
    """Simple image/volume -> (array [nz, ny, nx] or [ny, nx], header)."""
    h, order = read_header(path)
    nx, ny, nz, labbyt = _geom(h)
    if int(h[23]) != 0:
        raise ValueError(f"{path}: is a stack; use read_stack")
    with open(path, "rb") as f:
        f.seek(labbyt)
        d = np.frombuffer(f.read(nx * ny * nz * 4), dtype=order + "f4").astype(np.float32)
    if d.size != nx * ny * nz:
        raise ValueError(f"{path}: truncated data")
    d = d.reshape(nz, ny, nx)
    return (d[0] if nz == 1 and int(h[4]) == 1 else d), h


def write_image(path, arr, *, angles=None):
    """Write a 2-D image (IFORM 1) or 3-D volume (IFORM 3) as a simple file."""
    a = np.ascontiguousarray(arr, dtype="<f4")
    if a.ndim == 2:
        nz, (ny, nx), iform = 1, a.shape, 1
    elif a.ndim == 3:
        (nz, ny, nx), iform = a.shape, 3
    else:
        raise ValueError("2-D or 3-D array expected")
    h = _make_header(nx, ny, nz, iform, data=a, angles=angles)
    with open(path, "wb") as f:
        f.write(h.astype("<f4").tobytes())
        f.write(a.tobytes())


def read_stack(path, numbers=None):
    """Stack or indexed stack file -> (array [n, ny, nx], list of image
    numbers, per-image headers).  numbers None: every image (1..MAXIM; for
    an indexed stack every number present in the index)."""
    h, order = read_header(path)
    nx, ny, nz, labbyt = _geom(h)
    istack, maxim = int(h[23]), int(h[25])
    if istack == 0:
        raise ValueError(f"{path}: not a stack")
    per = labbyt + nx * ny * nz * 4
    index = None
    base = labbyt
    if istack < 0:   # indexed stack: MAXINDX = -ISTACK, then the index records
        maxindx = -istack
        indxrec = -(-maxindx // nx)
        with open(path, "rb") as f:
            f.seek(labbyt)
            index = np.frombuffer(f.read(indxrec * nx * 4), dtype=order + "i4")[:maxindx].astype(np.int64)
        base = labbyt + indxrec * nx * 4
        if numbers is None:
            numbers = [int(k) + 1 for k in np.nonzero(index > 0)[0]]
    nums = list(range(1, maxim + 1)) if numbers is None else list(numbers)
    out = np.zeros((len(nums), ny, nx) if nz == 1 else (len(nums), nz, ny, nx), np.float32)
    heads = []
    with open(path, "rb") as f:
        for i, k in enumerate(nums):
            if index is not None:
                if k < 1 or k > len(index) or index[k - 1] <= 0:
                    raise ValueError(f"{path}: image {k} not in the indexed stack")
                slot = int(index[k - 1])
            else:
                if k < 1 or k > maxim:
                    raise ValueError(f"{path}: image {k} not in stack (MAXIM {maxim})")
                slot = k
            f.seek(base + (slot - 1) * per)
            ih = np.frombuffer(f.read(labbyt), dtype=order + "f4").astype(np.float32)
            d = np.frombuffer(f.read(nx * ny * nz * 4), dtype=order + "f4").astype(np.float32)
            out[i] = d.reshape(out.shape[1:])
            heads.append(ih)
    return out, nums, heads


def write_stack(path, arr, *, angles=None, numbers=None, maxindx=None):
    """Write images [n, ny, nx] as a stack (numbers 1..n); optional angles [n, 3].
    With ``numbers`` (and ``maxindx`` >= max(numbers)) an indexed stack is
    written instead: image i gets number numbers[i] and storage slot i+1."""
    a = np.ascontiguousarray(arr, dtype="<f4")
    n, ny, nx = a.shape
    iform = 1
    nums = list(range(1, n + 1)) if numbers is None else [int(k) for k in numbers]
    with open(path, "wb") as f:
        if numbers is None:
            f.write(_make_header(nx, ny, 1, iform, istack=2, maxim=n).astype("<f4").tobytes())
        else:
            maxindx = int(maxindx if maxindx is not None else max(nums))
            if len(nums) != n or min(nums) < 1 or max(nums) > maxindx or len(set(nums)) != n:
                raise ValueError("indexed stack: numbers must be distinct, in 1..maxindx")
            h = _make_header(nx, ny, 1, iform, istack=0, maxim=max(nums))
            h[23] = -maxindx            # ISTACK = -MAXINDX
            h[27] = n                   # LASTINDX: highest storage slot in use
            f.write(h.astype("<f4").tobytes())
            indxrec = -(-maxindx // nx)
            index = np.zeros(indxrec * nx, "<i4")
            for slot, k in enumerate(nums, start=1):
                index[k - 1] = slot
            f.write(index.tobytes())
        for i in range(n):
            ang = None if angles is None else angles[i]
            f.write(_make_header(nx, ny, 1, iform, istack=0, imgnum=nums[i], data=a[i],
                                 angles=ang).astype("<f4").tobytes())
            f.write(a[i].tobytes())


# ----------------------------------------------------------------- doc files
def read_doc(path):
    """Document file -> {key: np.array(registers)} (comment lines skipped)."""
    out = {}
    with open(path) as f:
        for line in f:
            if len(line) > 1 and line[1] == ";" or line.lstrip().startswith(";"):
                continue
            parts = line.split()
            if len(parts) < 2:
                continue
            try:
                key = int(parts[0])
                nreg = int(parts[1])
            except ValueError:
                continue
            vals = [float(v) for v in parts[2:2 + nreg]]
            out[key] = np.array(vals, np.float64)
    return out


def write_doc(path, rows, comment="", keys=None):
    """rows: iterable of register lists; keys default to 1..n."""
    rows = [list(r) for r in rows]
    keys = list(range(1, len(rows) + 1)) if keys is None else list(keys)
    with open(path, "w") as f:
        stamp = datetime.datetime.now().strftime("%d-%b-%Y AT %H:%M:%S").upper()
        f.write(f" ; {comment}   {stamp}   {os.path.basename(path)}\n")
        for k, r in zip(keys, rows):
            f.write(f"{k:6d} {len(r):2d} " + " ".join(f"{v:12.6g}" for v in r) + "\n")


# ----------------------------------------------------------------- names
def parse_numbers(spec: str):
    """SPIDER file-number list '1-12,15,20-22' -> [1..12, 15, 20, 21, 22]."""
    out = []
    for part in re.split(r"[,\s]+", spec.strip()):
        if not part:
            continue
        m = re.fullmatch(r"(-?\d+)-(\d+)", part)
        if m:
            a, b = int(m.group(1)), int(m.group(2))
            out.extend(range(a, b + 1))
        else:
            out.append(int(part))
    return out


def expand_template(template: str, number: int) -> str:
    """'jnk***' + 7 -> 'jnk007'; 'stk@***' + 7 -> 'stk@007' (asterisks = digits)."""
    m = re.search(r"\*+", template)
    if not m:
        return template
    w = m.end() - m.start()
    return template[:m.start()] + f"{number:0{w}d}" + template[m.end():]


def add_extension(name: str, ext: str = "spi") -> str:
    base = name.split("@")[0]
    if os.path.splitext(base)[1]:
        return name
    if "@" in name:
        a, b = name.split("@", 1)
        return f"{a}.{ext}@{b}"
    return f"{name}.{ext}"


def read_images(template: str, numbers, ext: str = "spi"):
    """Images named by a template ('jnk***' or 'stk@***') and file numbers -> [n, ny, nx]."""
    t = add_extension(template, ext)
    if "@" in t:
        path = t.split("@", 1)[0]
        imgs, _, _ = read_stack(path, numbers)
        return imgs
    arrs = [read_image(expand_template(t, k))[0] for k in numbers]
    return np.stack(arrs).astype(np.float32)


# ----------------------------------------------------------------- streaming
class ImageSource:
    """The images named by a template and file numbers ('jnk***' files or a
    'stk@***' stack / indexed stack), read by position without loading them
    all: ``shape`` = (ny, nx); ``read_into(start, out)`` fills out[:count]
    with images numbers[start:start+count]."""

    def __init__(self, template: str, numbers, ext: str = "spi"):
        self.numbers = list(numbers)
        if not self.numbers:
            raise ValueError("no images")
        t = add_extension(template, ext)
        self.stack = "@" in t
        if self.stack:
            self.path = t.split("@", 1)[0]
            h, self.order = read_header(self.path)
            nx, ny, nz, labbyt = _geom(h)
            if nz != 1:
                raise ValueError(f"{self.path}: stack of volumes, images expected")
            istack = int(h[23])
            if istack == 0:
                raise ValueError(f"{self.path}: not a stack")
            self._per = labbyt + nx * ny * 4
            self._labbyt = labbyt
            self._base = labbyt
            self._slot = {}
            if istack < 0:
                maxindx = -istack
                indxrec = -(-maxindx // nx)
                with open(self.path, "rb") as f:
                    f.seek(labbyt)
                    index = np.frombuffer(f.read(indxrec * nx * 4), dtype=self.order + "i4")[:maxindx]
                self._base = labbyt + indxrec * nx * 4
                for k in self.numbers:
                    if k < 1 or k > len(index) or index[k - 1] <= 0:
                        raise ValueError(f"{self.path}: image {k} not in the indexed stack")
                    self._slot[k] = int(index[k - 1])
            else:
                maxim = int(h[25])
                for k in self.numbers:
                    if k < 1 or k > maxim:
                        raise ValueError(f"{self.path}: image {k} not in stack (MAXIM {maxim})")
                    self._slot[k] = k
        else:
            self.template = t
            h, _ = read_header(expand_template(t, self.numbers[0]))
            nx, ny, _, _ = _geom(h)
        self.shape = (ny, nx)

    def __len__(self):
        return len(self.numbers)

    def read_into(self, start: int, out: np.ndarray) -> int:
        """Read up to len(out) images from position start into out; returns the count."""
        ny, nx = self.shape
        count = min(len(out), len(self.numbers) - start)
        if not self.stack:
            for i in range(count):
                img, _ = read_image(expand_template(self.template, self.numbers[start + i]))
                if img.shape != (ny, nx):
                    raise ValueError(f"image {self.numbers[start + i]}: size {img.shape} differs from {(ny, nx)}")
                out[i] = img
            return count
        with open(self.path, "rb", buffering=0) as f:
            for i in range(count):
                f.seek(self._base + (self._slot[self.numbers[start + i]] - 1) * self._per + self._labbyt)
                dst = out[i]
                if f.readinto(memoryview(dst).cast("B")) != nx * ny * 4:
                    raise ValueError(f"{self.path}: truncated data")
                if self.order == ">":
                    dst.byteswap(inplace=True)
        return count


def stream_images(src: "ImageSource", chunk: int, buffers=None):
    """Yield (start, images[count, ny, nx]) chunk by chunk.  The next chunk is
    read on a background thread while the caller works on the current one, so
    reading overlaps the caller's compute (for example a GPU insertion called
    through ctypes, which releases the GIL).  A yielded array is valid until
    the generator is resumed twice; ``buffers`` may pass two preallocated
    float32 arrays [chunk, ny, nx] (pinned host memory, for instance)."""
    from concurrent.futures import ThreadPoolExecutor
    ny, nx = src.shape
    n = len(src)
    chunk = max(1, min(int(chunk), n))
    if buffers is None:
        buffers = [np.empty((chunk, ny, nx), np.float32) for _ in range(2)]
    with ThreadPoolExecutor(max_workers=1) as pool:
        pending = pool.submit(src.read_into, 0, buffers[0][:chunk])
        start, i = 0, 0
        while start < n:
            count = pending.result()
            cur = buffers[i % 2]
            nxt = start + count
            if nxt < n:
                pending = pool.submit(src.read_into, nxt, buffers[(i + 1) % 2][:chunk])
            yield start, cur[:count]
            start, i = nxt, i + 1
