// The mixed-precision factor's update matrices, U = -L21 L21^T in FP32 by 3xTF32 on the
// 5th-generation tensor cores: TMA copies of K-major operand tiles into shared memory,
// tcgen05.mma kind::tf32 into a TMEM accumulator, tcgen05.ld in the epilogue.
//
// Before a level's products, pack_tc_kernel writes each supernode's L21 once as a K-major FP32
// array P (row i of L21 = row i of P: [hi(0..wpad) | lo(0..wpad)], wpad = w rounded up to 32,
// hi = x rounded to TF32 and lo = x - hi, exact in FP32; the padding is zero); likewise, at the
// end of an outer block of panels, the block's columns below it for the updates past the block. The tensor core
// then reads hi exactly, and hi hi + hi lo + lo hi keeps FP32 accuracy (the 3xTF32 split) with no
// per-tile conversion work.
//
// syrk_tc_kernel: one CTA of 128 threads per tile of up to 128 x 128 outputs. Thread 0 is the
// producer: per K chunk of 16 it issues four 2D TMA loads (A hi, A lo, B hi, B lo: boxes of
// 128 rows x 64 bytes, 64-byte swizzle, rows past the end zero-filled) into a three-stage ring
// (97 KB: two CTAs share an SM, one's loads and epilogue beside the other's MMAs), completing on
// the stage's "full" mbarrier. Thread 32 issues the chunk's 2 x 3 MMAs (M 128, N 128, K 8 each)
// and commits them to the stage's "empty" mbarrier, which the producer waits on
// before refilling the stage. A diagonal tile (A = B) loads one operand pair. All four warps then
// read the accumulator (warp q owns TMEM lanes 32q..32q+31, the tile's rows) and write C. Every
// wait is bounded by time: a wait that gives up records DeviceStatus::timeout, and the CTA drains
// the copies still in flight (again bounded) and frees its TMEM before returning.
#include <cstdint>

#include "kernels.cuh"

namespace fc {

namespace {

constexpr int TC_M = 128, TC_N = 128, TC_KC = TC_KBOX, TC_THREADS = 128, TC_COLS = 128;
constexpr int TILE_BYTES = TC_M * TC_KC * 4;             // one operand tile of a chunk (8 KB)
constexpr int STAGE_BYTES = 4 * TILE_BYTES;              // A hi, A lo, B hi, B lo
constexpr int STAGES = 3;
constexpr size_t TC_SMEM = STAGES * STAGE_BYTES + 1024;  // + alignment slack: two CTAs fit on an SM
constexpr unsigned long long WAIT_NS = 2000000000ull;    // a wait longer than 2 s gives up
constexpr int TMAP_BYTES = 128;                          // sizeof(CUtensorMap)
static_assert(TC_M == GEMM_TC_M && TC_N == GEMM_TC_N && TC_KPAD % TC_KC == 0 && TC_KC * 4 == 64, "tile shape");

// instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory operand descriptor of a K-major tile with 64-byte swizzle (what the TMA writes
// for 64-byte rows): 8-row atoms of 512 bytes (SBO), LBO unused (1), version 1, layout type 4.
// A step of 8 K values inside the atom adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
         (4ull << 61);
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
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 2D tile load (x = the K element, a multiple of 16 here; y = the row) completing on `bar`
__device__ __forceinline__ void tma_load(void *dst, const void *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
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

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem),
      "l"(a), "l"(b), "r"(IDESC), "r"(accumulate));
}

__global__ void __launch_bounds__(TC_THREADS, 2) syrk_tc_kernel(const TcTask *__restrict__ tasks,
                                                                const unsigned char *__restrict__ maps,
                                                                DeviceStatus *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char tc_raw[];
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_fail;
  __shared__ int s_issued;  // chunks whose copies the producer issued
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  const TcTask task = tasks[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nq = (task.K + TC_KC - 1) / TC_KC;
  const bool diag = task.bi == task.bj;
  const void *map = maps + (size_t)task.map * TMAP_BYTES;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&full[i]);
      mbar_init(&empty[i]);
    }
    s_fail = 0;
    s_issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    // the tensor map was written to global memory before the launch
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int wpad = task.wpad;
  const uint32_t bytes = diag ? 2 * TILE_BYTES : STAGE_BYTES;
  if (tid == 0) {
    // producer
    int q = 0;
    for (; q < nq && !s_fail; ++q) {
      const int s = q % STAGES;
      if (q >= STAGES && !mbar_wait(&empty[s], ((q / STAGES) - 1) & 1)) {
        s_fail = 1;
        break;
      }
      unsigned char *st = base + s * STAGE_BYTES;
      const int kc = q * TC_KC;
      mbar_expect(&full[s], bytes);
      tma_load(st, map, kc, task.bi, &full[s]);
      tma_load(st + TILE_BYTES, map, wpad + kc, task.bi, &full[s]);
      if (!diag) {
        tma_load(st + 2 * TILE_BYTES, map, kc, task.bj, &full[s]);
        tma_load(st + 3 * TILE_BYTES, map, wpad + kc, task.bj, &full[s]);
      }
    }
    s_issued = q;
  } else if (tid == 32) {
    // MMA issuer
    for (int q = 0; q < nq; ++q) {
      const int s = q % STAGES;
      if (s_fail || !mbar_wait(&full[s], (q / STAGES) & 1)) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_hi = smem_u32(base + s * STAGE_BYTES), a_lo = a_hi + TILE_BYTES;
      const uint32_t b_hi = diag ? a_hi : a_hi + 2 * TILE_BYTES, b_lo = diag ? a_lo : a_hi + 3 * TILE_BYTES;
#pragma unroll
      for (int k8 = 0; k8 < TC_KC / 8; ++k8) {
        const uint32_t step = k8 * 32;  // 8 FP32 values along K inside the 64-byte swizzle atom
        const uint64_t ah = smem_desc(a_hi + step), al = smem_desc(a_lo + step);
        const uint64_t bh = smem_desc(b_hi + step), bl = smem_desc(b_lo + step);
        mma_tf32(tmem, ah, bh, (q > 0 || k8 > 0) ? 1u : 0u);
        mma_tf32(tmem, ah, bl, 1u);
        mma_tf32(tmem, al, bh, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&empty[s]))
                   : "memory");
    }
  }
  __syncthreads();
  // the last chunk's commit covers every MMA issued before it
  if (tid == 0 && nq > 0 && !s_fail) {
    const int q = nq - 1;
    if (!mbar_wait(&empty[q % STAGES], (q / STAGES) & 1)) s_fail = 1;
  }
  if (tid == 0 && s_fail) {
    // drain: the copies still in flight (at most the last STAGES chunks issued: the producer
    // refills a stage only after its MMAs are done) land before the shared memory goes away
    for (int q = max(0, s_issued - STAGES); q < s_issued; ++q) mbar_wait(&full[q % STAGES], (q / STAGES) & 1);
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (s_fail) {
    if (tid == 0) atomicExch(&status->timeout, 1u);
  } else {
    const bool lower = task.flags & 1, store = task.flags & 2;
    float *C = task.C;
    const int64_t c_sj = task.c_sj;
    const int i = warp * 32 + lane;  // this thread's row = its TMEM lane
    for (int c0 = 0; c0 < TC_N; c0 += 32) {
      float v[32];
      if (nq > 0) {
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] = 0.f;
      }
      if (i < task.M) {
        float old[32];
        if (!store) {
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const int j = c0 + c;
            old[c] = j < task.N && (!lower || i >= j) ? C[i + (int64_t)j * c_sj] : 0.f;
          }
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int j = c0 + c;
          if (j < task.N && (!lower || i >= j)) C[i + (int64_t)j * c_sj] = store ? -v[c] : old[c] - v[c];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_COLS));
}

// P rows [r0, r0 + TC_PACK_ROWS), columns [k0, k1), of a block of supernode s's L (FP32 in the L
// arena, column-major): hi and lo as K-major rows, through a shared tile so that both the reads
// (down a column) and the writes (along a row) are coalesced.
__global__ void __launch_bounds__(256) pack_tc_kernel(Tree t, const PackTask *__restrict__ tasks,
                                                       float *__restrict__ P) {
  __shared__ float tile[TC_KPAD][TC_PACK_ROWS + 1];
  const PackTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int m = t.height[s], u = m - task.row0, w = task.kw;
  // Lb[k m + i] = L(row0 + i, c0 + k)
  const float *Lb = static_cast<const float *>(t.L) + t.loff[s] + (int64_t)task.c0 * m + task.row0;
  const int r0 = task.r0, nr = min(TC_PACK_ROWS, u - r0), wpad = task.wpad;
  float *Pp = P + task.poff;
  for (int kc = task.k0; kc < task.k1; kc += TC_KPAD) {
    for (int e = threadIdx.x; e < TC_KPAD * TC_PACK_ROWS; e += blockDim.x) {
      const int k = e / TC_PACK_ROWS, r = e - k * TC_PACK_ROWS;
      tile[k][r] = kc + k < w && r < nr ? Lb[(int64_t)(kc + k) * m + r0 + r] : 0.f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TC_KPAD * TC_PACK_ROWS; e += blockDim.x) {
      const int r = e / TC_KPAD, k = e - r * TC_KPAD;
      if (r < nr) {
        const float x = tile[k][r];
        uint32_t h;
        asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(x));
        const float hi = __uint_as_float(h);
        float *row = Pp + (int64_t)(r0 + r) * 2 * wpad;
        row[kc + k] = hi;
        row[wpad + kc + k] = x - hi;
      }
    }
    __syncthreads();
  }
}

}  // namespace

void launch_syrk_tc(const TcTask *tasks, const void *maps, int count, DeviceStatus *status, cudaStream_t st) {
  if (count <= 0) return;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(syrk_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    configured = true;
  }
  syrk_tc_kernel<<<count, TC_THREADS, TC_SMEM, st>>>(tasks, static_cast<const unsigned char *>(maps), status);
}

void launch_pack_tc(const Tree &t, const PackTask *tasks, float *P, int count, cudaStream_t st) {
  if (count > 0) pack_tc_kernel<<<count, 256, 0, st>>>(t, tasks, P);
}

}  // namespace fc
