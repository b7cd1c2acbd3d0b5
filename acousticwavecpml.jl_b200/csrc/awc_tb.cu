// awc_tb.cu — instantiations and launch wrappers of the two-step 3D kernel
// (awc_tb.cuh). Kept in its own translation unit so it compiles in parallel
// with the rest of the library.
#include "awc_tb.cuh"

namespace awc {

namespace {
template <typename T, typename I, bool XY>
void* kernel_of() {
  return reinterpret_cast<void*>(step3d_tb<T, I, TB_ROWS, TB_STAGES, XY>);
}
}  // namespace

template <typename T>
cudaError_t tb_launch(const TbParams<T>& P, bool xy, bool i64, const CUtensorMap& mpt,
                      const CUtensorMap& mpo, const CUtensorMap& mf, unsigned nblocks,
                      cudaStream_t st) {
  if (nblocks == 0) return cudaSuccess;
  constexpr int smem = tb_smem<T, TB_ROWS, TB_STAGES>();
  const dim3 grid(nblocks), block(32 * TB_ROWS);
  if (xy) {
    if (i64)
      step3d_tb<T, int64_t, TB_ROWS, TB_STAGES, true><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
    else
      step3d_tb<T, int32_t, TB_ROWS, TB_STAGES, true><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
  } else {
    if (i64)
      step3d_tb<T, int64_t, TB_ROWS, TB_STAGES, false><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
    else
      step3d_tb<T, int32_t, TB_ROWS, TB_STAGES, false><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
  }
  return cudaGetLastError();
}

template cudaError_t tb_launch<float>(const TbParams<float>&, bool, bool, const CUtensorMap&,
                                      const CUtensorMap&, const CUtensorMap&, unsigned,
                                      cudaStream_t);
template cudaError_t tb_launch<double>(const TbParams<double>&, bool, bool, const CUtensorMap&,
                                       const CUtensorMap&, const CUtensorMap&, unsigned,
                                       cudaStream_t);

cudaError_t tb_init_attrs() {
  void* const kf[4] = {kernel_of<float, int32_t, false>(), kernel_of<float, int32_t, true>(),
                       kernel_of<float, int64_t, false>(), kernel_of<float, int64_t, true>()};
  void* const kd[4] = {kernel_of<double, int32_t, false>(), kernel_of<double, int32_t, true>(),
                       kernel_of<double, int64_t, false>(), kernel_of<double, int64_t, true>()};
  for (void* k : kf) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tb_smem<float, TB_ROWS, TB_STAGES>());
    if (e != cudaSuccess) return e;
  }
  for (void* k : kd) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tb_smem<double, TB_ROWS, TB_STAGES>());
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int tb_occupancy(bool f64, bool xy) {
  int occ = 0;
  if (f64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, xy ? kernel_of<double, int32_t, true>() : kernel_of<double, int32_t, false>(),
        32 * TB_ROWS, tb_smem<double, TB_ROWS, TB_STAGES>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, xy ? kernel_of<float, int32_t, true>() : kernel_of<float, int32_t, false>(),
        32 * TB_ROWS, tb_smem<float, TB_ROWS, TB_STAGES>());
  cudaGetLastError();
  return occ > 0 ? occ : 1;
}

}  // namespace awc
