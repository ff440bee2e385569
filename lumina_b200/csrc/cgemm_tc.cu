// cgemm_tc.cu -- Y = A X for many right-hand sides of a cached FP32 matrix on
// the sm_100a tensor cores (tcgen05, TMA, TMEM).
//
// The reference applies the cached matrix one vector at a time
// (MatvecSession::matvec, backend.rs:54; matvec.wgsl:19-39).  With many
// right-hand sides (polarisations, incidence directions) the product is a
// dense complex GEMM and belongs on the tensor cores.
//
// Real formulation.  The interleaved complex FP32 matrix A (dim x ld complex,
// row-major) is read in place as a real K-major operand Ar[dim][K], K = 2 ld:
// Ar[m][2c] = Re A[m][c], Ar[m][2c+1] = Im A[m][c].  The right-hand sides
// become a real K-major operand Bt[2R][K] with
//   Bt[2r][2c]   =  Re X[c][r],   Bt[2r][2c+1]   = -Im X[c][r],
//   Bt[2r+1][2c] =  Im X[c][r],   Bt[2r+1][2c+1] =  Re X[c][r],
// so D = Ar Bt^T holds Re Y[m][r] in column 2r and Im Y[m][r] in column 2r+1.
//
// Precision (3xTF32).  A TF32 operand keeps 10 explicit mantissa bits.  Each
// FP32 value v is split as v = hi + lo with hi = v with its low 13 mantissa
// bits cleared (exact in TF32) and lo = v - hi (exact in FP32), and
//   A B ~= Ahi Bhi + Ahi Blo + Alo Bhi
// (relative error ~2^-21 per product).  B is split when it is packed (from
// FP64 vectors); the A tile is split in shared memory after its TMA load, so
// A is read from HBM exactly once, in its stored form.  The tensor core's
// own FP32 accumulation drifts with the number of MMAs summed into one
// accumulator, so the K loop is cut into chains of kChain stages that
// alternate between two TMEM accumulators; while one chain runs, the
// epilogue warps add the previous one into FP32 registers
// (round-to-nearest), the CUDA-core accumulation an FP32 product would use.
//
// CTA (384 threads, one per SM: ~192 KB of shared memory):
//   warp 0      TMA producer: A tile 128 rows x 32 floats, B hi/lo tiles
//               NT rows x 32 floats, 128-byte swizzle, mbarrier per stage;
//   warp 1      MMA issuer: 12 tcgen05.mma (M=128, N=NT, K=8) per stage into
//               the current chain's accumulator; tcgen05.commit frees the
//               stage and, at a chain's end, hands the accumulator over;
//   warp 2      TMEM allocation (2 x NT FP32 columns) and release;
//   warps 4-11  split A into hi/lo in shared memory per stage, drain each
//               finished chain (tcgen05.ld, one TMEM lane = one matrix row
//               per thread, half of the columns per warp), write the result.
// Split-K over gridDim.z fills the 148 SMs when dim/128 x column tiles is
// small; the partial sums are reduced in FP64 in a fixed order.
//
// Every mbarrier wait is bounded by a clock64 deadline: on expiry the CTA
// records a status code, stops issuing work, waits (bounded) for its copies
// and MMAs in flight, releases TMEM and returns.  The host reports a
// nonzero status as LUM_ERR_TIMEOUT.  The pipeline waits use a limit passed
// at launch (kWaitCycles, ~2 s, unless LUMINA_TC_WAIT_CYCLES sets another
// positive count of SM clocks); the final waits for the copies and MMAs in
// flight always use kWaitCycles, so a short pipeline limit never lets the
// CTA release shared memory or TMEM under an operation that has not landed.
// LUMINA_TC_WITHHOLD_SPLIT=1 makes the first CTA's split warps withhold their
// arrival on the first stage, so that its MMA issuer's wait runs out: the
// check that a wait which never completes ends with TIMEOUT and leaves the
// context usable.
#include "lumina_internal.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>

namespace lum {
namespace {

constexpr int kTcM = 128;            // matrix rows per CTA = TMEM lanes
constexpr int kTcBK = 32;            // FP32 K elements per stage (one 128-byte row)
constexpr int kTcWorkers = 256;     // split / drain / epilogue threads (warps 4-11)
constexpr int kTcThreads = 128 + kTcWorkers;
// Stages per accumulation chain.  The tensor core's FP32 accumulation loses
// accuracy with the length of a chain (measured: ~1e-4 relative after ~7000
// MMAs into one accumulator); chains of two stages (24 MMAs) are drained into
// registers and summed there with round-to-nearest FP32 adds.
constexpr int kChain = 2;
constexpr int kATileBytes = kTcM * 128;
constexpr uint32_t kTf32Mask = 0xffffe000u;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

template <int NT> struct TcCfg {
  static constexpr int kBTileBytes = NT * 128;
  static constexpr int kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;
  static constexpr int kStages = (NT >= 256) ? 2 : (NT >= 128 ? 3 : (NT >= 32 ? 4 : 5));
  static constexpr int kTmemCols = 2 * (NT < 32 ? 32 : NT);  // two chain accumulators
  // tiles + 1 KB alignment slack + barriers / TMEM slot / abort flag
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 256;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
      : "memory");
  return ok != 0;
}

// Waits for the phase of `parity` to complete.  Gives up when `abort` is set
// by another role or after `limit` SM clocks (then sets *abort and the status).
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort, int* status,
                          int code, long long limit) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (abort && *abort) return false;
    if (clock64() - t0 > limit) {
      if (abort) *abort = 1;
      atomicCAS(status, 0, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 128 bytes, 8-row groups 1024 bytes apart (tile base 1024-byte aligned).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);  // start address
  d |= (uint64_t)1 << 16;                           // leading offset (unused: swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                 // stride offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                           // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                           // SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  // load and wait in one statement: no use of r[] can be scheduled before the wait
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr)
      : "memory");
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, M = 128, N = NT.
template <int NT> __device__ __forceinline__ uint32_t idesc_tf32() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NT >> 3) << 17) |
         ((uint32_t)(kTcM >> 4) << 24);
}

template <int NT>
__global__ void __launch_bounds__(kTcThreads, 1)
cgemm_tf32x3_kernel(const __grid_constant__ CUtensorMap map_a,
                    const __grid_constant__ CUtensorMap map_bhi,
                    const __grid_constant__ CUtensorMap map_blo, int dim, int ktiles,
                    int ktiles_per_split, int nrhs, double2* __restrict__ Y, long long syc,
                    long long syr, float2* __restrict__ part, int* __restrict__ status,
                    long long wait_cycles, int withhold) {
  using C = TcCfg<NT>;
  constexpr int S = C::kStages;
  constexpr int CPT = NT / 2;  // accumulator columns per epilogue thread
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char* sA = smem;
  unsigned char* sAlo = sA + S * kATileBytes;
  unsigned char* sBhi = sAlo + S * kATileBytes;
  unsigned char* sBlo = sBhi + S * C::kBTileBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(sBlo + S * C::kBTileBytes);
  uint64_t* split = full + S;
  uint64_t* empty = split + S;
  uint64_t* acc_full = empty + S;    // [2]: a chain's MMAs have completed
  uint64_t* acc_empty = acc_full + 2;  // [2]: the chain's accumulator has been drained
  uint64_t* done = acc_empty + 2;      // every MMA of the CTA has completed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTcM;
  const int n0 = blockIdx.y * NT;
  const int kt0 = blockIdx.z * ktiles_per_split;
  const int nk = min(ktiles, kt0 + ktiles_per_split) - kt0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&split[s], kTcWorkers);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kTcWorkers);
    }
    mbar_init(done, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"((uint32_t)C::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    int it = 0;
    for (; it < nk; ++it) {
      const int s = it % S;
      const uint32_t ph = (it / S) & 1;
      if (*abort) break;
      if (it >= S && !mbar_wait(&empty[s], ph ^ 1u, abort, status, 1, wait_cycles)) break;
      mbar_expect_tx(&full[s], kATileBytes + 2 * C::kBTileBytes);
      const int kx = (kt0 + it) * kTcBK;
      tma_load_2d(sA + s * kATileBytes, &map_a, kx, m0, &full[s]);
      tma_load_2d(sBhi + s * C::kBTileBytes, &map_bhi, kx, n0, &full[s]);
      tma_load_2d(sBlo + s * C::kBTileBytes, &map_blo, kx, n0, &full[s]);
    }
    // copies still in flight must land before the CTA's shared memory is released
    for (int q = max(0, it - S); q < it; ++q)
      mbar_wait(&full[q % S], (q / S) & 1, nullptr, status, 2, kWaitCycles);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer.  Chain c (kChain stages) accumulates into TMEM buffer
    // c & 1; the epilogue warps drain it while chain c + 1 runs.
    const uint32_t idesc = idesc_tf32<NT>();
    for (int it = 0; it < nk; ++it) {
      const int s = it % S;
      const uint32_t ph = (it / S) & 1;
      const int c = it / kChain;
      const bool first = (it % kChain) == 0;
      const uint32_t acc = tmem + (uint32_t)((c & 1) * NT);
      if (first && c >= 2 &&
          !mbar_wait(&acc_empty[c & 1], ((c >> 1) - 1) & 1, abort, status, 6, wait_cycles))
        break;
      if (!mbar_wait(&split[s], ph, abort, status, 3, wait_cycles)) break;
      tc_fence_after();
      const uint32_t a = smem_u32(sA + s * kATileBytes);
      const uint32_t alo = smem_u32(sAlo + s * kATileBytes);
      const uint32_t bh = smem_u32(sBhi + s * C::kBTileBytes);
      const uint32_t bl = smem_u32(sBlo + s * C::kBTileBytes);
#pragma unroll
      for (int kk = 0; kk < kTcBK / 8; ++kk) {  // K = 8 TF32 = 32 bytes per MMA
        const uint64_t dA = smem_desc(a + 32 * kk), dAlo = smem_desc(alo + 32 * kk);
        const uint64_t dBh = smem_desc(bh + 32 * kk), dBl = smem_desc(bl + 32 * kk);
        mma_tf32(acc, dA, dBh, idesc, (first && kk == 0) ? 0u : 1u);
        mma_tf32(acc, dA, dBl, idesc, 1u);
        mma_tf32(acc, dAlo, dBh, idesc, 1u);
      }
      mma_commit(&empty[s]);
      if ((it % kChain) == kChain - 1 || it == nk - 1) mma_commit(&acc_full[c & 1]);
    }
    // no MMA may be in flight when TMEM is released (also after an abort)
    mma_commit(done);
    mbar_wait(done, 0, nullptr, status, 7, kWaitCycles);
  } else if (warp >= 4) {
    // ---- split A into TF32 hi / lo; drain finished chains into registers;
    // write the result.  Warp 4 + 4h + q owns TMEM lanes 32q.. (rows) and
    // accumulator columns [h NT/2, (h + 1) NT/2).
    const int t = threadIdx.x - 128;
    const int quarter = warp & 3, half = (warp - 4) >> 2;
    const uint32_t lane_base = (uint32_t)(32 * quarter) << 16;
    float sum[CPT];
#pragma unroll
    for (int e = 0; e < CPT; ++e) sum[e] = 0.f;
    bool ok = true;
    auto drain = [&](int c) {
      if (!mbar_wait(&acc_full[c & 1], (c >> 1) & 1, abort, status, 5, wait_cycles)) {
        ok = false;
        return;
      }
      tc_fence_after();
      const uint32_t base = tmem + lane_base + (uint32_t)((c & 1) * NT + half * CPT);
#pragma unroll
      for (int cb = 0; cb < CPT / 8; ++cb) {
        uint32_t r[8];
        tmem_ld8(base + 8 * cb, r);
#pragma unroll
        for (int e = 0; e < 8; ++e) sum[8 * cb + e] += __uint_as_float(r[e]);
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[c & 1]);
    };
    for (int it = 0; it < nk && ok; ++it) {
      const int s = it % S;
      const uint32_t ph = (it / S) & 1;
      if (!mbar_wait(&full[s], ph, abort, status, 4, wait_cycles)) {
        ok = false;
        break;
      }
      uint4* a = reinterpret_cast<uint4*>(sA + s * kATileBytes);
      uint4* alo = reinterpret_cast<uint4*>(sAlo + s * kATileBytes);
#pragma unroll
      for (int c = 0; c < kATileBytes / 16 / kTcWorkers; ++c) {
        const int q = t + kTcWorkers * c;
        const uint4 v = a[q];
        const uint4 h = make_uint4(v.x & kTf32Mask, v.y & kTf32Mask, v.z & kTf32Mask,
                                   v.w & kTf32Mask);
        const uint4 l = make_uint4(
            __float_as_uint(__uint_as_float(v.x) - __uint_as_float(h.x)),
            __float_as_uint(__uint_as_float(v.y) - __uint_as_float(h.y)),
            __float_as_uint(__uint_as_float(v.z) - __uint_as_float(h.z)),
            __float_as_uint(__uint_as_float(v.w) - __uint_as_float(h.w)));
        a[q] = h;
        alo[q] = l;
      }
      // make these generic-proxy writes visible to the tensor core (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (!(withhold && it == 0 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0))
        mbar_arrive(&split[s]);
      // the chain before the one this stage starts is complete: drain it
      if (it % kChain == 0 && it > 0) drain(it / kChain - 1);
    }
    if (ok && nk > 0) drain((nk - 1) / kChain);
    if (ok && !*abort) {
      const int row = m0 + 32 * quarter + lane;
      if (row < dim) {
#pragma unroll
        for (int e = 0; e < CPT / 2; ++e) {
          const int rhs = (n0 + half * CPT) / 2 + e;
          if (rhs < nrhs) {
            if (part)
              part[((size_t)blockIdx.z * nrhs + rhs) * dim + row] =
                  make_float2(sum[2 * e], sum[2 * e + 1]);
            else
              Y[(long long)row * syc + (long long)rhs * syr] =
                  make_double2(sum[2 * e], sum[2 * e + 1]);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)C::kTmemCols)
                 : "memory");
  }
}

// Bt hi/lo rows (K-major, 2 ld floats per row) from the FP64 right-hand sides.
__global__ void tc_pack_b(int dim, int ld, int nrhs, int npad, const double2* __restrict__ X,
                          long long sxc, long long sxr, float2* __restrict__ bhi,
                          float2* __restrict__ blo) {
  const size_t total = (size_t)npad * ld;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(q / ld), c = (int)(q % ld);
    const int r = n >> 1;
    double v0 = 0.0, v1 = 0.0;
    if (r < nrhs && c < dim) {
      const double2 x = X[(long long)c * sxc + (long long)r * sxr];
      if (n & 1) {
        v0 = x.y;
        v1 = x.x;
      } else {
        v0 = x.x;
        v1 = -x.y;
      }
    }
    const float h0 = __uint_as_float(__float_as_uint((float)v0) & kTf32Mask);
    const float h1 = __uint_as_float(__float_as_uint((float)v1) & kTf32Mask);
    bhi[q] = make_float2(h0, h1);
    blo[q] = make_float2((float)(v0 - (double)h0), (float)(v1 - (double)h1));
  }
}

// Y[row, r] = sum over splits of the partials, in split order, in FP64.
__global__ void tc_reduce(int dim, int nrhs, int ksplit, const float2* __restrict__ part,
                          double2* __restrict__ Y, long long syc, long long syr) {
  const size_t total = (size_t)nrhs * dim;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(q / dim), row = (int)(q % dim);
    double sx = 0.0, sy = 0.0;
    for (int z = 0; z < ksplit; ++z) {
      const float2 p = part[(size_t)z * total + q];
      sx += p.x;
      sy += p.y;
    }
    Y[(long long)row * syc + (long long)r * syr] = make_double2(sx, sy);
  }
}

using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

// 2D FP32 map over rows x K (K innermost), box 32 x box_rows, 128-byte swizzle.
lum_status make_map(void* out, const void* base, size_t k, size_t rows, int box_rows) {
  EncodeFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return LUM_ERR_UNAVAILABLE;
  }
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(k * sizeof(float))};
  cuuint32_t box[2] = {(cuuint32_t)kTcBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                   const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return LUM_ERR_DEVICE;
  }
  return LUM_OK;
}

template <int NT>
lum_status launch_tc(CachedOperator& op, int nrhs, int mt, int nt, int ksplit, int kps,
                     double2* Y, long long syc, long long syr, cudaStream_t st) {
  using C = TcCfg<NT>;
  LUM_TRY_CUDA(cudaFuncSetAttribute(cgemm_tf32x3_kernel<NT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, C::kSmemBytes));
  TcWork& w = op.tc;
  const int ktiles = (int)(2 * op.ld / kTcBK);
  const CUtensorMap* ma = reinterpret_cast<const CUtensorMap*>(w.map_a);
  const CUtensorMap* mh = reinterpret_cast<const CUtensorMap*>(w.map_bhi);
  const CUtensorMap* ml = reinterpret_cast<const CUtensorMap*>(w.map_blo);
  float2* part = ksplit > 1 ? w.part.as<float2>() : nullptr;
  long long wait_cycles = kWaitCycles;
  if (const char* env = std::getenv("LUMINA_TC_WAIT_CYCLES")) {
    const long long v = std::atoll(env);
    if (v > 0) wait_cycles = v;
  }
  const char* wh = std::getenv("LUMINA_TC_WITHHOLD_SPLIT");
  const int withhold = (wh && wh[0] == '1') ? 1 : 0;
  cgemm_tf32x3_kernel<NT><<<dim3(mt, nt, ksplit), kTcThreads, C::kSmemBytes, st>>>(
      *ma, *mh, *ml, op.dim, ktiles, kps, nrhs, Y, syc, syr, part, w.status.as<int>(),
      wait_cycles, withhold);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

}  // namespace

lum_status cgemm_tf32x3(CachedOperator& op, const double2* X, long long sxc, long long sxr,
                        double2* Y, long long syc, long long syr, int nrhs, cudaStream_t st) {
  if (op.precision != LUM_FP32) {
    set_error("the tensor-core product needs FP32 matrix storage");
    return LUM_ERR_INVALID;
  }
  TcWork& w = op.tc;
  const int cols = 2 * nrhs;
  int NT = 16;
  while (NT < cols && NT < 256) NT *= 2;
  const int nt = (cols + NT - 1) / NT;
  const int npad = nt * NT;
  const int mt = (op.dim + kTcM - 1) / kTcM;
  const int ktiles = (int)(2 * op.ld / kTcBK);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Split K so that the grid fills whole waves of one CTA per SM: the
  // smallest split whose last wave is >= 90 % full (else the fullest), each
  // split keeping >= 16 stages.
  const int kmax = std::max(1, std::min(16, ktiles / 16));
  int ksplit = 1;
  double best = 0.0;
  for (int ks = 1; ks <= kmax; ++ks) {
    const int ctas = mt * nt * ks;
    const double eff = (double)ctas / ((double)sms * ((ctas + sms - 1) / sms));
    if (eff > best + 1e-9) {
      best = eff;
      ksplit = ks;
    }
    if (eff >= 0.9) break;
  }
  const int kps = (ktiles + ksplit - 1) / ksplit;
  ksplit = (ktiles + kps - 1) / kps;

  if (!w.status.p) {
    LUM_TRY(w.status.alloc(sizeof(int)));
    LUM_TRY_CUDA(cudaMemsetAsync(w.status.p, 0, sizeof(int), st));
  }
  if (w.mapped_a != op.A.p) {
    LUM_TRY(make_map(w.map_a, op.A.p, 2 * op.ld, (size_t)op.dim, kTcM));
    w.mapped_a = op.A.p;
  }
  if (w.npad != npad) {
    const size_t bytes = sizeof(float) * (size_t)npad * 2 * op.ld;
    LUM_TRY(w.bhi.alloc(bytes));
    LUM_TRY(w.blo.alloc(bytes));
    LUM_TRY(make_map(w.map_bhi, w.bhi.p, 2 * op.ld, (size_t)npad, NT));
    LUM_TRY(make_map(w.map_blo, w.blo.p, 2 * op.ld, (size_t)npad, NT));
    w.npad = npad;
  }
  if (ksplit > 1) {
    const size_t pb = sizeof(float2) * (size_t)ksplit * nrhs * op.dim;
    if (w.part_bytes < pb) {
      LUM_TRY(w.part.alloc(pb));
      w.part_bytes = pb;
    }
  }
  const size_t packs = (size_t)npad * op.ld;
  tc_pack_b<<<(unsigned)std::min<size_t>((packs + 255) / 256, 8192), 256, 0, st>>>(
      op.dim, (int)op.ld, nrhs, npad, X, sxc, sxr, w.bhi.as<float2>(), w.blo.as<float2>());
  LUM_CHECK_LAUNCH();
  switch (NT) {
    case 16: LUM_TRY(launch_tc<16>(op, nrhs, mt, nt, ksplit, kps, Y, syc, syr, st)); break;
    case 32: LUM_TRY(launch_tc<32>(op, nrhs, mt, nt, ksplit, kps, Y, syc, syr, st)); break;
    case 64: LUM_TRY(launch_tc<64>(op, nrhs, mt, nt, ksplit, kps, Y, syc, syr, st)); break;
    case 128: LUM_TRY(launch_tc<128>(op, nrhs, mt, nt, ksplit, kps, Y, syc, syr, st)); break;
    default: LUM_TRY(launch_tc<256>(op, nrhs, mt, nt, ksplit, kps, Y, syc, syr, st)); break;
  }
  if (ksplit > 1) {
    const size_t total = (size_t)nrhs * op.dim;
    tc_reduce<<<(unsigned)std::min<size_t>((total + 255) / 256, 8192), 256, 0, st>>>(
        op.dim, nrhs, ksplit, w.part.as<float2>(), Y, syc, syr);
    LUM_CHECK_LAUNCH();
  }
  return LUM_OK;
}

// Nonzero when a pipeline wait of an earlier product gave up (reset on read).
lum_status cgemm_status(CachedOperator& op, cudaStream_t st) {
  if (!op.tc.status.p) return LUM_OK;
  int h = 0;
  LUM_TRY_CUDA(cudaMemcpyAsync(&h, op.tc.status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  if (h) {
    LUM_TRY_CUDA(cudaMemsetAsync(op.tc.status.p, 0, sizeof(int), st));
    set_error("tensor-core product: pipeline wait %d timed out", h);
    return LUM_ERR_TIMEOUT;
  }
  return LUM_OK;
}

}  // namespace lum
