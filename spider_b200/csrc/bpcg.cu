// BP CG (linear interpolation) -- kernels land in the next revision.
#include "../../include/spider_b200.h"
#include "ctx.h"
namespace spi {
void cg_release(spi_ctx* c) { for (auto& b : c->cg_buf) b.release(); }
}
using namespace spi;
extern "C" {
int spi_bpcg(spi_ctx*, const float*, int, int, const float*, float, float, float, int, int, float, float*, float*, int*) {
  return fail(kInvalid, "spi_bpcg: not built in this revision");
}
int spi_cg_project(spi_ctx*, const float*, int, float, const float*, int, float*, int) {
  return fail(kInvalid, "spi_cg_project: not built in this revision");
}
int spi_cg_backproject(spi_ctx*, const float*, int, float, const float*, int, float*, int) {
  return fail(kInvalid, "spi_cg_backproject: not built in this revision");
}
}
