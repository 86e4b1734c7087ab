// TMA (cp.async.bulk.tensor) tile loads with mbarrier completion, for the
// x-pass kernels.  A spectral field set (ncomp components of Nx rows x
// Ny*(Nz/2+1) columns, back to back) is viewed as one 2-D tensor of
// ncomp*Nx rows and Ny*Hz columns of 8-byte units (one complex64, or half of
// a complex128); its row pitch Ny*Hz*8 B is a multiple of 16 B for even Ny.
// Boxes are CW columns (CW*8 >= 16 B, tile starts at multiples of CW, so the
// innermost coordinate times 8 B is a multiple of 16 B) by up to 256 rows.
// Out-of-range columns of a ragged last tile are filled with zeros.
// Loads only; no cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ts {

// ----------------------------------------------------------------------------
// device side
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `polls` polls (default 2^22; each try_wait may
// suspend briefly), sets the timeout bit of *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int polls = 1 << 22) {
  for (int i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 1);
  return false;
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size multiple of 16)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// 2-D tiled load of box {x: columns (8-byte units), y: rows} at (x, y) into dst
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace ts

namespace ts {
// ----------------------------------------------------------------------------
// host side: 2-D tensor map of a field set (see the file comment)
// ----------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// map over the rows_total x cols complex matrix at `base` (8-byte units: `units`
// per complex); box of `cw` complex columns by `rows` rows
inline cudaError_t make_field_map(CUtensorMap* m, const void* base, long long cols, long long rows_total,
                                  int units, int cw, int rows) {
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return cudaErrorMisalignedAddress;
  const cuuint64_t dims[2] = {(cuuint64_t)(cols * units), (cuuint64_t)rows_total};
  const cuuint64_t strides[1] = {(cuuint64_t)(cols * units * 8)};
  const cuuint32_t box[2] = {(cuuint32_t)(cw * units), (cuuint32_t)rows};
  const cuuint32_t estr[2] = {1, 1};
  if ((strides[0] & 15) != 0 || ((cuuint64_t)box[0] * 8) % 16 != 0) return cudaErrorInvalidValue;
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
}  // namespace ts
