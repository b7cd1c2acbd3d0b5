// awc_tb.cu — instantiations and launch wrappers of the two-step 3D kernel
// (awc_tb.cuh). Kept in its own translation unit so it compiles in parallel
// with the rest of the library.
#include "awc_tb.cuh"

namespace awc {

namespace {
template <typename T, typename I, int W, bool XY>
void* kernel_of() {
  return reinterpret_cast<void*>(step3d_tb<T, I, W, TB_STAGES, XY>);
}

template <typename T, int W>
cudaError_t launch_w(const TbParams<T>& P, bool xy, bool i64, const CUtensorMap& mpt,
                     const CUtensorMap& mpo, const CUtensorMap& mf, unsigned nblocks,
                     cudaStream_t st) {
  constexpr int smem = tb_smem<T, W, TB_STAGES>();
  const dim3 grid(nblocks), block(32 * W);
  if (xy) {
    if (i64)
      step3d_tb<T, int64_t, W, TB_STAGES, true><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
    else
      step3d_tb<T, int32_t, W, TB_STAGES, true><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
  } else {
    if (i64)
      step3d_tb<T, int64_t, W, TB_STAGES, false><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
    else
      step3d_tb<T, int32_t, W, TB_STAGES, false><<<grid, block, smem, st>>>(mpt, mpo, mf, P);
  }
  return cudaGetLastError();
}

template <typename T, int W>
cudaError_t attrs_w() {
  void* const k[4] = {kernel_of<T, int32_t, W, false>(), kernel_of<T, int32_t, W, true>(),
                      kernel_of<T, int64_t, W, false>(), kernel_of<T, int64_t, W, true>()};
  for (void* f : k) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               tb_smem<T, W, TB_STAGES>());
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T, int W>
int occ_w(bool xy) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, xy ? kernel_of<T, int32_t, W, true>() : kernel_of<T, int32_t, W, false>(), 32 * W,
      tb_smem<T, W, TB_STAGES>());
  cudaGetLastError();
  return occ > 0 ? occ : 1;
}
}  // namespace

template <typename T>
cudaError_t tb_launch(const TbParams<T>& P, bool xy, bool i64, int rows, const CUtensorMap& mpt,
                      const CUtensorMap& mpo, const CUtensorMap& mf, unsigned nblocks,
                      cudaStream_t st) {
  if (nblocks == 0) return cudaSuccess;
  if (rows == 8) return launch_w<T, 8>(P, xy, i64, mpt, mpo, mf, nblocks, st);
  if (rows == 16) return launch_w<T, 16>(P, xy, i64, mpt, mpo, mf, nblocks, st);
  return cudaErrorInvalidValue;
}

template cudaError_t tb_launch<float>(const TbParams<float>&, bool, bool, int, const CUtensorMap&,
                                      const CUtensorMap&, const CUtensorMap&, unsigned,
                                      cudaStream_t);
template cudaError_t tb_launch<double>(const TbParams<double>&, bool, bool, int,
                                       const CUtensorMap&, const CUtensorMap&, const CUtensorMap&,
                                       unsigned, cudaStream_t);

cudaError_t tb_init_attrs() {
  cudaError_t e;
  if ((e = attrs_w<float, 8>()) != cudaSuccess || (e = attrs_w<float, 16>()) != cudaSuccess ||
      (e = attrs_w<double, 8>()) != cudaSuccess || (e = attrs_w<double, 16>()) != cudaSuccess)
    return e;
  return cudaSuccess;
}

int tb_occupancy(bool f64, bool xy, int rows) {
  if (f64) return rows == 8 ? occ_w<double, 8>(xy) : occ_w<double, 16>(xy);
  return rows == 8 ? occ_w<float, 8>(xy) : occ_w<float, 16>(xy);
}

}  // namespace awc
