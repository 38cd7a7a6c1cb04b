// C -= A B^T (and the other GemmTask forms) in FP32 by 3xTF32 on the 5th-generation tensor cores:
// tcgen05.mma kind::tf32 from shared-memory operand descriptors into a TMEM accumulator.
//
// One CTA of 256 threads per task tile of up to 128 x 128 outputs (M = 128 rows of A, N = 128
// rows of B). K advances in chunks of 32 through a three-stage ring. cp.async copies each chunk's FP32
// operands (A and B with unit row stride: the factor's column-major panels) straight into the
// canonical K-major, no-swizzle layout (8-row x 16-byte core matrices), two chunks ahead. The
// threads round each value in place to TF32 (hi, which the tensor core then reads exactly) and
// write the "lo" tiles, lo = x - hi (exact in FP32), and thread 0 issues the chunk's 4 x 3 MMAs (hi hi + hi lo + lo hi; M 128, N 128, K 8 each),
// committed to the stage's mbarrier; a stage is refilled once its MMAs are done. The epilogue
// reads the accumulator with tcgen05.ld (warps w and w + 4 own TMEM lanes 32w..32w+31, the rows,
// one half of the 128 columns each) and writes C. Every mbarrier wait is bounded
// (DeviceStatus::timeout records a wait that gave up).
#include <cstdint>

#include "kernels.cuh"

namespace fc {

namespace {

constexpr int TC_M = 128, TC_N = 128, TC_KC = 32, TC_THREADS = 256, TC_COLS = 128;
constexpr int A_BYTES = TC_M * TC_KC * 4, B_BYTES = TC_N * TC_KC * 4;  // one operand tile of a chunk
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;                  // A hi, A lo, B hi, B lo
constexpr int STAGES = 3;
constexpr size_t TC_SMEM = STAGES * STAGE_BYTES + 1024;                  // + 1 KB alignment slack
constexpr unsigned long long WAIT_NS = 2000000000ull;                    // a wait longer than 2 s gives up

// instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory operand descriptor, K-major without swizzle: core matrices of 8 rows x 16 bytes,
// the next core matrix along K at LBO = 128 bytes, along M/N at SBO = 1024 bytes (a chunk's 32 K
// values per row group), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46);
}
// byte offset of element (row, k) of a chunk tile in that layout
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)));
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for phase `parity` of the mbarrier to complete; false after WAIT_NS.
__device__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  while (!mbar_try(bar, parity))
    if (now_ns() - t0 > WAIT_NS) return false;
  return true;
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp4(void *smem, const void *gmem, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(ok ? 4 : 0));
}

__global__ void __launch_bounds__(TC_THREADS, 1) gemm_tc_kernel(const GemmTask *__restrict__ tasks,
                                                                DeviceStatus *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char tc_raw[];
  __shared__ __align__(8) uint64_t bars[STAGES];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  const GemmTask *tp = tasks + blockIdx.x;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M = tp->M, N = tp->N, K = tp->K;
  const float *A = static_cast<const float *>(tp->A);
  const float *B = static_cast<const float *>(tp->B);
  const int64_t a_sk = tp->a_sk, b_sk = tp->b_sk;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < STAGES; ++i) mbar_init(&bars[i]);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int nq = (K + TC_KC - 1) / TC_KC;
  // copies: row tid % 128 of A and of B for k = (tid / 128) * 16 + 0..15 (a warp: 32 consecutive
  // rows of one k, coalesced)
  const int ar = tid & 127, ak0 = (tid >> 7) * 16, br = ar, bk0 = ak0;
  auto issue = [&](int q) {
    if (q < nq) {
      unsigned char *st = base + (q % STAGES) * STAGE_BYTES;
      const int kc = q * TC_KC, kk = min(TC_KC, K - kc);
#pragma unroll
      for (int k = ak0; k < ak0 + 16; ++k) {
        const bool ok = ar < M && k < kk;
        cp4(st + tile_off(ar, k), ok ? A + ar + (int64_t)(kc + k) * a_sk : A, ok);
      }
#pragma unroll
      for (int k = bk0; k < bk0 + 16; ++k) {
        const bool ok = br < N && k < kk;
        cp4(st + 2 * A_BYTES + tile_off(br, k), ok ? B + br + (int64_t)(kc + k) * b_sk : B, ok);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);  // an empty group past the end keeps the count uniform
  };
  // x -> (hi, lo): hi = x rounded to TF32 (so the tensor core's reading of it drops nothing),
  // lo = x - hi (exact in FP32)
  auto split = [](float v, float &hi, float &lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(v));
    hi = __uint_as_float(h);
    lo = v - hi;
  };
  issue(0);
  issue(1);
  for (int q = 0; q < nq; ++q) {
    const int s = q % STAGES;
    unsigned char *st = base + s * STAGE_BYTES;
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // chunk q has landed (this thread's copies)
    __syncthreads();
    if (s_fail) break;  // every thread reads the same value after the barrier
    // hi in place and the lo tiles: 16-byte groups (4 consecutive k of one row); A: 1024, B: 1024
    for (int g = tid; g < (A_BYTES + B_BYTES) / 16; g += TC_THREADS) {
      const int off = g < A_BYTES / 16 ? g * 16 : A_BYTES + g * 16;  // A hi | A lo | B hi | B lo
      const float4 x = *reinterpret_cast<const float4 *>(st + off);
      float4 hi, lo;
      split(x.x, hi.x, lo.x);
      split(x.y, hi.y, lo.y);
      split(x.z, hi.z, lo.z);
      split(x.w, hi.w, lo.w);
      *reinterpret_cast<float4 *>(st + off) = hi;
      *reinterpret_cast<float4 *>(st + off + (g < A_BYTES / 16 ? A_BYTES : B_BYTES)) = lo;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_hi = smem_u32(st), a_lo = a_hi + A_BYTES, b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
      for (int k8 = 0; k8 < TC_KC / 8; ++k8) {
        const uint32_t step = k8 * 256;  // K = 8 values = two core matrices along K
        const uint64_t ah = smem_desc(a_hi + step), al = smem_desc(a_lo + step);
        const uint64_t bh = smem_desc(b_hi + step), bl = smem_desc(b_lo + step);
        const uint32_t acc0 = (q > 0 || k8 > 0) ? 1u : 0u;
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                tmem),
            "l"(ah), "l"(bh), "r"(IDESC), "r"(acc0));
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                tmem),
            "l"(ah), "l"(bl), "r"(IDESC), "r"(1u));
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                tmem),
            "l"(al), "l"(bh), "r"(IDESC), "r"(1u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&bars[s]))
                   : "memory");
    }
    // refill the stage of chunk q - 1 (chunk q + 2) once its MMAs are done
    if (q + 2 < nq && q >= 1) {
      const int sp = (q - 1) % STAGES;
      if (!mbar_wait(&bars[sp], ((q - 1) / STAGES) & 1)) s_fail = 1;  // benign race: all store 1
    }
    issue(q + 2);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // the last chunk's commit covers every MMA issued before it
  if (nq > 0 && !s_fail) {
    const int q = nq - 1;
    if (!mbar_wait(&bars[q % STAGES], (q / STAGES) & 1)) s_fail = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (s_fail) {
    if (tid == 0) atomicExch(&status->timeout, 1u);
  } else {
    const bool lower = tp->flags & 1, store = tp->flags & 2, partial = tp->flags & 4;
    float *C = static_cast<float *>(tp->C);
    const int64_t c_si = tp->c_si, c_sj = tp->c_sj;
    const int quad = warp & 3, half = warp >> 2;
    const int i = quad * 32 + lane;  // this thread's row = its TMEM lane
    for (int part = 0; part < 2; ++part) {
      const int c0 = half * 64 + part * 32;
      float v[32];
      if (nq > 0) {
        tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + c0, v);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] = 0.f;
      }
      if (i < M) {
        float old[32];
        if (!partial && !store) {
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const int j = c0 + c;
            old[c] = j < N && (!lower || i >= j) ? C[i * c_si + (int64_t)j * c_sj] : 0.f;
          }
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int j = c0 + c;
          if (j < N && (!lower || i >= j))
            C[i * c_si + (int64_t)j * c_sj] = partial ? v[c] : store ? -v[c] : old[c] - v[c];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_COLS));
}

}  // namespace

void launch_gemm_tc(const GemmTask *tasks, int count, DeviceStatus *status, cudaStream_t st) {
  if (count <= 0) return;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    configured = true;
  }
  gemm_tc_kernel<<<count, TC_THREADS, TC_SMEM, st>>>(tasks, status);
}

}  // namespace fc
