// flsp_k_sep2.cu — separable stage kernel, 2D instances.
#include "flsp_k_sep.cuh"
#include "flsp_tables.h"

namespace flsp {

int upload_tables_sep2() {
  cudaError_t e = upload_tables_here();
  if (e != cudaSuccess) return set_error(FLSP_ERR_CUDA, std::string("tables: ") + cudaGetErrorString(e));
  return FLSP_OK;
}

int sep2_call(int what, const Ctx& c, const VelDev* v, const int* tile, size_t* bytes, const void* in,
              const void* phin, void* out, const DevClock* clk, int stage, int combine, double ct_explicit) {
  return sep_call<2>(what, c, v, tile, bytes, in, phin, out, clk, stage, combine, ct_explicit);
}

}  // namespace flsp
