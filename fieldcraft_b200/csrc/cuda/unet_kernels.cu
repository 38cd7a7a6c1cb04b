// Kernels of the learned preconditioner (see unet_kernels.cuh): 3x3x3 convolutions as implicit
// GEMMs on the BF16 tensor pipe (ldmatrix fragments, mma m16n8k16, FP32 accumulation), their
// weight gradients as GEMMs over voxels with a fixed-order reduction, grid transfers, Adam, and
// the FP64 vector kernels of flexible CG.
#include <algorithm>
#include <cstdint>

#include "unet_kernels.cuh"

namespace fc {
namespace unet {

namespace {

using bf16 = __nv_bfloat16;
constexpr int THREADS = 128;
constexpr float SLOPE = 0.05f;  // leaky ReLU: x for x > 0, SLOPE x otherwise
__device__ __forceinline__ float gate(float mask) { return mask > 0.f ? 1.f : SLOPE; }
constexpr int TX = 8, TY = 8;         // output tile of a convolution CTA: 8 x 8 voxels of one z plane
constexpr int HX = TX + 2, HY = TY + 2, HV = HX * HY * 3;  // its input halo

__device__ __forceinline__ void cp16(void *smem, const void *gmem, bool ok) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(ok ? 16 : 0));
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void *p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void *p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
// D = A B + D, A 16 x 16 (row major), B 16 x 8 (column major), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__host__ __device__ constexpr int cstride(int c) { return c + 8; }  // shared-memory channel stride
template <int CIN, int COUT>
__host__ __device__ constexpr size_t conv_smem() {
  return sizeof(bf16) * ((size_t)27 * COUT * cstride(CIN) + (size_t)HV * cstride(CIN));
}

// One CTA per 8 x 8 tile of a z plane (persistent over tiles); all 27 taps' weights stay in
// shared memory. Warp w computes voxel rows y = 2w, 2w + 1 (16 voxels) x COUT channels.
template <int CIN, int COUT>
__global__ void __launch_bounds__(THREADS) conv3_kernel(Grid g, const bf16 *__restrict__ in,
                                                       const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                       int relu, const bf16 *__restrict__ mask, bf16 *__restrict__ out) {
  constexpr int CS = cstride(CIN);
  extern __shared__ __align__(16) unsigned char smem[];
  bf16 *ws = reinterpret_cast<bf16 *>(smem);
  bf16 *ts = ws + 27 * COUT * CS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tg = lane & 3;
  for (int e = tid; e < 27 * COUT * (CIN / 8); e += THREADS) {
    const int row = e / (CIN / 8), c8 = e % (CIN / 8);
    cp16(ws + row * CS + c8 * 8, w + row * CIN + c8 * 8, true);
  }
  commit();
  const int ntx = (g.X + TX - 1) / TX, nty = (g.Y + TY - 1) / TY;
  const int ntiles = ntx * nty * g.Z;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x0 = (tile % ntx) * TX, y0 = ((tile / ntx) % nty) * TY, z = tile / (ntx * nty);
    __syncthreads();
    for (int e = tid; e < HV * (CIN / 8); e += THREADS) {
      const int hv = e / (CIN / 8), c8 = e % (CIN / 8);
      const int hx = hv % HX, hy = (hv / HX) % HY, hz = hv / (HX * HY);
      const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z + hz - 1;
      const bool ok = gx >= 0 && gx < g.X && gy >= 0 && gy < g.Y && gz >= 0 && gz < g.Z;
      const int64_t v = ok ? ((int64_t)gz * g.Y + gy) * g.X + gx : 0;
      cp16(ts + hv * CS + c8 * 8, in + v * CIN + c8 * 8, ok);
    }
    commit();
    wait_all();
    __syncthreads();
    float acc[COUT / 8][4];
#pragma unroll
    for (int nt = 0; nt < COUT / 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    const int q = lane >> 3, r = lane & 7;
    for (int tap = 0; tap < 27; ++tap) {
      const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
      // A rows: voxel (x = r, y = 2 warp + (q & 1)); B rows: output channel
      const bf16 *arow = ts + (((1 + dz) * HY + (1 + 2 * warp + (q & 1) + dy)) * HX + (1 + r + dx)) * CS + (q >> 1) * 8;
#pragma unroll
      for (int ks = 0; ks < CIN / 16; ++ks) {
        uint32_t a[4];
        ldsm_x4(a, arow + ks * 16);
#pragma unroll
        for (int np = 0; np < COUT / 16; ++np) {
          uint32_t b[4];
          const int co = (2 * np + (q >> 1)) * 8 + r;
          ldsm_x4(b, ws + (tap * COUT + co) * CS + ks * 16 + (q & 1) * 8);
          mma_bf16(acc[2 * np], a, b[0], b[1]);
          mma_bf16(acc[2 * np + 1], a, b[2], b[3]);
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gx = x0 + gq, gy = y0 + 2 * warp + h;
      if (gx >= g.X || gy >= g.Y) continue;
      const int64_t v = ((int64_t)z * g.Y + gy) * g.X + gx;
#pragma unroll
      for (int nt = 0; nt < COUT / 8; ++nt) {
        const int co = nt * 8 + 2 * tg;
        float v0 = acc[nt][2 * h], v1 = acc[nt][2 * h + 1];
        if (bias) v0 += bias[co], v1 += bias[co + 1];
        if (relu) v0 = v0 > 0.f ? v0 : SLOPE * v0, v1 = v1 > 0.f ? v1 : SLOPE * v1;
        if (mask) {
          const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162 *>(mask + v * COUT + co);
          v0 *= gate(__bfloat162float(mk.x));
          v1 *= gate(__bfloat162float(mk.y));
        }
        *reinterpret_cast<__nv_bfloat162 *>(out + v * COUT + co) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

// Weight gradient: CTA (chunk, tap group of 4): warp w accumulates tap 4 group + w over the
// chunk's tiles as the GEMM dW_tap (COUT x CIN) += dY^T (COUT x voxels) X_tap (voxels x CIN), both
// operands read transposed by ldmatrix.trans from channels-last tiles.
template <int CIN, int COUT>
__host__ __device__ constexpr size_t dw_smem() {
  return sizeof(bf16) * ((size_t)HV * cstride(CIN) + (size_t)TX * TY * cstride(COUT));
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(THREADS) conv3_dw_kernel(Grid g, const bf16 *__restrict__ in,
                                                          const bf16 *__restrict__ dy, int tiles_per_chunk,
                                                          float *__restrict__ part) {
  constexpr int CS = cstride(CIN), DS = cstride(COUT);
  extern __shared__ __align__(16) unsigned char smem[];
  bf16 *ts = reinterpret_cast<bf16 *>(smem);
  bf16 *ds = ts + HV * CS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tg = lane & 3, q = lane >> 3, r = lane & 7;
  const int tap = blockIdx.y * 4 + warp;
  const bool active = tap < 27;
  const int dx = tap % 3 - 1, dyo = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
  const int ntx = (g.X + TX - 1) / TX, nty = (g.Y + TY - 1) / TY;
  const int ntiles = ntx * nty * g.Z;
  float acc[COUT / 16][CIN / 8][4];
#pragma unroll
  for (int mt = 0; mt < COUT / 16; ++mt)
#pragma unroll
    for (int nt = 0; nt < CIN / 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.f;
  const int t0 = blockIdx.x * tiles_per_chunk, t1 = min(ntiles, t0 + tiles_per_chunk);
  for (int tile = t0; tile < t1; ++tile) {
    const int x0 = (tile % ntx) * TX, y0 = ((tile / ntx) % nty) * TY, z = tile / (ntx * nty);
    __syncthreads();
    for (int e = tid; e < HV * (CIN / 8); e += THREADS) {
      const int hv = e / (CIN / 8), c8 = e % (CIN / 8);
      const int hx = hv % HX, hy = (hv / HX) % HY, hz = hv / (HX * HY);
      const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z + hz - 1;
      const bool ok = gx >= 0 && gx < g.X && gy >= 0 && gy < g.Y && gz >= 0 && gz < g.Z;
      const int64_t v = ok ? ((int64_t)gz * g.Y + gy) * g.X + gx : 0;
      cp16(ts + hv * CS + c8 * 8, in + v * CIN + c8 * 8, ok);
    }
    for (int e = tid; e < TX * TY * (COUT / 8); e += THREADS) {
      const int m = e / (COUT / 8), c8 = e % (COUT / 8);
      const int gx = x0 + m % TX, gy = y0 + m / TX;
      const bool ok = gx < g.X && gy < g.Y;
      const int64_t v = ok ? ((int64_t)z * g.Y + gy) * g.X + gx : 0;
      cp16(ds + m * DS + c8 * 8, dy + v * COUT + c8 * 8, ok);
    }
    commit();
    wait_all();
    __syncthreads();
    if (!active) continue;
#pragma unroll
    for (int ks = 0; ks < TX * TY / 16; ++ks) {
      uint32_t a[COUT / 16][4];
#pragma unroll
      for (int mt = 0; mt < COUT / 16; ++mt)  // rows: voxel ks 16 + (q >> 1) 8 + r; columns: channel
        ldsm_x4_t(a[mt], ds + (ks * 16 + (q >> 1) * 8 + r) * DS + mt * 16 + (q & 1) * 8);
      const int k = ks * 16 + (q & 1) * 8 + r;  // B row: voxel k of the tile, shifted by the tap
      const bf16 *brow = ts + (((1 + dz) * HY + (1 + k / TX + dyo)) * HX + (1 + k % TX + dx)) * CS;
#pragma unroll
      for (int np = 0; np < CIN / 16; ++np) {
        uint32_t b[4];
        ldsm_x4_t(b, brow + (2 * np + (q >> 1)) * 8);
#pragma unroll
        for (int mt = 0; mt < COUT / 16; ++mt) {
          mma_bf16(acc[mt][2 * np], a[mt], b[0], b[1]);
          mma_bf16(acc[mt][2 * np + 1], a[mt], b[2], b[3]);
        }
      }
    }
  }
  if (!active) return;
  float *dst = part + ((int64_t)blockIdx.x * 27 + tap) * COUT * CIN;
#pragma unroll
  for (int mt = 0; mt < COUT / 16; ++mt)
#pragma unroll
    for (int nt = 0; nt < CIN / 8; ++nt) {
      const int co = mt * 16 + gq, ci = nt * 8 + 2 * tg;
      dst[co * CIN + ci] = acc[mt][nt][0];
      dst[co * CIN + ci + 1] = acc[mt][nt][1];
      dst[(co + 8) * CIN + ci] = acc[mt][nt][2];
      dst[(co + 8) * CIN + ci + 1] = acc[mt][nt][3];
    }
}

__global__ void dw_reduce_kernel(int chunks, int64_t per_chunk, const float *__restrict__ part, float *__restrict__ gw) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < per_chunk; e += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < chunks; ++c) s += part[(int64_t)c * per_chunk + e];
    gw[e] = s;
  }
}

// gb[c] = sum over voxels of dy[v][c]: CTA b sums its voxel range (4 lanes per channel, each a
// stride-4 sequence, combined in order); then one CTA sums the CTAs' partials in order.
constexpr int BIAS_CTAS = 256;
__global__ void __launch_bounds__(128) bias_part_kernel(int64_t voxels, int cout, const bf16 *__restrict__ dy,
                                                        float *__restrict__ part) {
  __shared__ float s[128];
  const int c = threadIdx.x % 32, lane4 = threadIdx.x / 32;
  const int64_t per = (voxels + gridDim.x - 1) / gridDim.x;
  const int64_t v0 = blockIdx.x * per, v1 = min(voxels, v0 + per);
  float acc = 0.f;
  if (c < cout)
    for (int64_t v = v0 + lane4; v < v1; v += 4) acc += __bfloat162float(dy[v * cout + c]);
  s[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < 32 && c < cout) part[blockIdx.x * 32 + c] = ((s[c] + s[32 + c]) + s[64 + c]) + s[96 + c];
}
__global__ void bias_reduce_kernel(int ctas, int cout, const float *__restrict__ part, float *__restrict__ gb) {
  const int c = threadIdx.x;
  if (c >= cout) return;
  float s = 0.f;
  for (int b = 0; b < ctas; ++b) s += part[b * 32 + c];
  gb[c] = s;
}

__global__ void flip_kernel(int cin, int cout, const bf16 *__restrict__ w, bf16 *__restrict__ wt) {
  const int total = 27 * cin * cout;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int ci = e % cin, co = (e / cin) % cout, tap = e / (cin * cout);
    wt[((26 - tap) * cin + ci) * cout + co] = w[e];
  }
}

__global__ void to_bf16_kernel(int64_t n, const float *__restrict__ src, bf16 *__restrict__ dst) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    dst[e] = __float2bfloat16_rn(src[e]);
}

constexpr int C32 = 32;
__global__ void pool_kernel(Grid gf, Grid gc, const bf16 *__restrict__ fine, bf16 *__restrict__ coarse) {
  const int64_t total = gc.voxels() * (C32 / 2);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % (C32 / 2)) * 2;
    const int64_t vc = e / (C32 / 2);
    const int x = (int)(vc % gc.X), y = (int)((vc / gc.X) % gc.Y), z = (int)(vc / ((int64_t)gc.X * gc.Y));
    float s0 = 0.f, s1 = 0.f;
    for (int k = 0; k < 8; ++k) {
      const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
      if (fx >= gf.X || fy >= gf.Y || fz >= gf.Z) continue;
      const __nv_bfloat162 f =
          *reinterpret_cast<const __nv_bfloat162 *>(fine + (((int64_t)fz * gf.Y + fy) * gf.X + fx) * C32 + c);
      s0 += __bfloat162float(f.x), s1 += __bfloat162float(f.y);
    }
    *reinterpret_cast<__nv_bfloat162 *>(coarse + vc * C32 + c) = __floats2bfloat162_rn(s0 * 0.125f, s1 * 0.125f);
  }
}

__global__ void up_add_kernel(Grid gf, Grid gc, const bf16 *__restrict__ coarse, const bf16 *__restrict__ skip,
                              bf16 *__restrict__ fine) {
  const int64_t total = gf.voxels() * (C32 / 2);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % (C32 / 2)) * 2;
    const int64_t v = e / (C32 / 2);
    const int x = (int)(v % gf.X), y = (int)((v / gf.X) % gf.Y), z = (int)(v / ((int64_t)gf.X * gf.Y));
    const int64_t vc = ((int64_t)(z / 2) * gc.Y + y / 2) * gc.X + x / 2;
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(coarse + vc * C32 + c);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(skip + v * C32 + c);
    *reinterpret_cast<__nv_bfloat162 *>(fine + v * C32 + c) = __floats2bfloat162_rn(
        __bfloat162float(a.x) + __bfloat162float(b.x), __bfloat162float(a.y) + __bfloat162float(b.y));
  }
}

__global__ void up_adjoint_kernel(Grid gf, Grid gc, const bf16 *__restrict__ dfine, const bf16 *__restrict__ mask,
                                  bf16 *__restrict__ dcoarse) {
  const int64_t total = gc.voxels() * (C32 / 2);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % (C32 / 2)) * 2;
    const int64_t vc = e / (C32 / 2);
    const int x = (int)(vc % gc.X), y = (int)((vc / gc.X) % gc.Y), z = (int)(vc / ((int64_t)gc.X * gc.Y));
    float s0 = 0.f, s1 = 0.f;
    for (int k = 0; k < 8; ++k) {
      const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
      if (fx >= gf.X || fy >= gf.Y || fz >= gf.Z) continue;
      const __nv_bfloat162 f =
          *reinterpret_cast<const __nv_bfloat162 *>(dfine + (((int64_t)fz * gf.Y + fy) * gf.X + fx) * C32 + c);
      s0 += __bfloat162float(f.x), s1 += __bfloat162float(f.y);
    }
    const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162 *>(mask + vc * C32 + c);
    s0 *= gate(__bfloat162float(mk.x));
    s1 *= gate(__bfloat162float(mk.y));
    *reinterpret_cast<__nv_bfloat162 *>(dcoarse + vc * C32 + c) = __floats2bfloat162_rn(s0, s1);
  }
}

__global__ void pool_adjoint_kernel(Grid gf, Grid gc, const bf16 *__restrict__ dcoarse, const bf16 *__restrict__ dskip,
                                    const bf16 *__restrict__ mask, bf16 *__restrict__ dfine) {
  const int64_t total = gf.voxels() * (C32 / 2);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % (C32 / 2)) * 2;
    const int64_t v = e / (C32 / 2);
    const int x = (int)(v % gf.X), y = (int)((v / gf.X) % gf.Y), z = (int)(v / ((int64_t)gf.X * gf.Y));
    const int64_t vc = ((int64_t)(z / 2) * gc.Y + y / 2) * gc.X + x / 2;
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(dcoarse + vc * C32 + c);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(dskip + v * C32 + c);
    const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162 *>(mask + v * C32 + c);
    const float s0 = (__bfloat162float(a.x) * 0.125f + __bfloat162float(b.x)) * gate(__bfloat162float(mk.x));
    const float s1 = (__bfloat162float(a.y) * 0.125f + __bfloat162float(b.y)) * gate(__bfloat162float(mk.y));
    *reinterpret_cast<__nv_bfloat162 *>(dfine + v * C32 + c) = __floats2bfloat162_rn(s0, s1);
  }
}

constexpr int CIO = 16;  // channels of the network's input and output grids
__global__ void scatter_input_kernel(Grid g, const int64_t *__restrict__ eq, const double *__restrict__ r,
                                     const float *__restrict__ feat, const double *__restrict__ scale,
                                     bf16 *__restrict__ x) {
  const int64_t total = g.voxels() * CIO;
  const double s = scale[0];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % CIO);
    const int64_t v = e / CIO;
    float val = 0.f;
    if (c < 3) {
      const int64_t q = eq[3 * v + c];
      if (q >= 0) val = (float)(r[q] * s);
    } else if (c == 3) {
      val = feat[v];
    }
    x[e] = __float2bfloat16_rn(val);
  }
}

__global__ void gather_output_kernel(Grid g, const int64_t *__restrict__ eq, const bf16 *__restrict__ y,
                                     const double *__restrict__ scale, double *__restrict__ z) {
  const int64_t total = g.voxels() * 3;
  const double s = scale[1];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = e / 3;
    const int c = (int)(e % 3);
    const int64_t q = eq[3 * v + c];
    if (q >= 0) z[q] = (double)__bfloat162float(y[v * CIO + c]) * s;
  }
}

__global__ void scatter_grad_kernel(Grid g, const int64_t *__restrict__ eq, const double *__restrict__ dz,
                                    const double *__restrict__ scale, bf16 *__restrict__ dy) {
  const int64_t total = g.voxels() * CIO;
  const double s = scale[1];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % CIO);
    const int64_t v = e / CIO;
    float val = 0.f;
    if (c < 3) {
      const int64_t q = eq[3 * v + c];
      if (q >= 0) val = (float)(dz[q] * s);
    }
    dy[e] = __float2bfloat16_rn(val);
  }
}

__global__ void adam_kernel(int64_t n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const float gr = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gr;
    const float vv = b2 * v[e] + (1.f - b2) * gr * gr;
    m[e] = mm, v[e] = vv;
    p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

// ---- FCG vectors --------------------------------------------------------------------------------
constexpr int DOT_CTAS = 296, MAX_PAIRS = 8;
struct PairPtrs {
  const double *a[MAX_PAIRS], *b[MAX_PAIRS];
};
__global__ void __launch_bounds__(256) dot_part_kernel(int64_t n, int pairs, PairPtrs pp, double *__restrict__ part) {
  __shared__ double s[256];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int k = 0; k < pairs; ++k) {
    double acc = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) acc += pp.a[k][i] * pp.b[k][i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[k * gridDim.x + blockIdx.x] = s[0];
    __syncthreads();
  }
}
__global__ void __launch_bounds__(256) dot_final_kernel(int ctas, int pairs, const double *__restrict__ part,
                                                        double *__restrict__ out) {
  __shared__ double s[256];
  for (int k = 0; k < pairs; ++k) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < ctas; b += blockDim.x) acc += part[k * ctas + b];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = s[0];
    __syncthreads();
  }
}

__global__ void axpy_dev_kernel(int64_t n, const double *__restrict__ alpha, double sign, const double *__restrict__ x,
                                double *__restrict__ y) {
  const double a = sign * alpha[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

struct DirPtrs {
  const double *p[MAX_PAIRS];
  int slot[MAX_PAIRS];  // where each direction's denominator p_j.q_j is kept
};
__global__ void fcg_direction_kernel(int64_t n, int m, const double *__restrict__ z, DirPtrs pj,
                                     const double *__restrict__ num, const double *__restrict__ den,
                                     double *__restrict__ p) {
  double beta[MAX_PAIRS];
  for (int j = 0; j < m; ++j) {
    const double d = den[pj.slot[j]];
    beta[j] = d != 0.0 ? num[j] / d : 0.0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = z[i];
    for (int j = 0; j < m; ++j) v -= beta[j] * pj.p[j][i];
    p[i] = v;
  }
}

__global__ void input_scales_kernel(int64_t n, const double *__restrict__ nrm2, double kref, double *__restrict__ s) {
  const double nr = sqrt(nrm2[0]);
  const double sn = sqrt((double)n);
  s[0] = nr > 0.0 ? sn / nr : 0.0;
  s[1] = nr / (sn * kref);
}

int grid_for(int64_t work) { return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 8)); }

template <int CIN, int COUT>
void conv3_launch(const Grid &g, const bf16 *in, const bf16 *w, const float *bias, bool relu, const bf16 *mask,
                  bf16 *out, cudaStream_t st) {
  static bool configured = false;
  constexpr size_t smem = conv_smem<CIN, COUT>();
  if (!configured) {
    cudaFuncSetAttribute(conv3_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  static int sms = 0, per = 1;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, conv3_kernel<CIN, COUT>, THREADS, smem);
    sms = std::max(sms, 1);
  }
  const int ntiles = ((g.X + TX - 1) / TX) * ((g.Y + TY - 1) / TY) * g.Z;
  const int grid = std::max(1, std::min(ntiles, sms * std::max(per, 1)));
  conv3_kernel<CIN, COUT><<<grid, THREADS, smem, st>>>(g, in, w, bias, relu ? 1 : 0, mask, out);
}

template <int CIN, int COUT>
void dw_launch(const Grid &g, const bf16 *in, const bf16 *dy, float *part, float *gw, cudaStream_t st) {
  static bool configured = false;
  constexpr size_t smem = dw_smem<CIN, COUT>();
  if (!configured) {
    cudaFuncSetAttribute(conv3_dw_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  const int ntiles = ((g.X + TX - 1) / TX) * ((g.Y + TY - 1) / TY) * g.Z;
  const int chunks = dw_chunks(g);
  const int per = (ntiles + chunks - 1) / chunks;
  conv3_dw_kernel<CIN, COUT><<<dim3(chunks, 7), THREADS, smem, st>>>(g, in, dy, per, part);
  const int64_t per_chunk = (int64_t)27 * CIN * COUT;
  dw_reduce_kernel<<<grid_for(per_chunk), 256, 0, st>>>(chunks, per_chunk, part, gw);
}

}  // namespace

void conv3(const Grid &g, int cin, int cout, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
           bool relu, const __nv_bfloat16 *mask, __nv_bfloat16 *out, cudaStream_t st) {
  if (cin == 32 && cout == 32)
    conv3_launch<32, 32>(g, in, w, bias, relu, mask, out, st);
  else if (cin == 16 && cout == 32)
    conv3_launch<16, 32>(g, in, w, bias, relu, mask, out, st);
  else if (cin == 32 && cout == 16)
    conv3_launch<32, 16>(g, in, w, bias, relu, mask, out, st);
  else
    conv3_launch<16, 16>(g, in, w, bias, relu, mask, out, st);
}

int dw_chunks(const Grid &g) {
  const int ntiles = ((g.X + TX - 1) / TX) * ((g.Y + TY - 1) / TY) * g.Z;
  return std::max(1, std::min(ntiles, 256));
}

void conv3_dw(const Grid &g, int cin, int cout, const __nv_bfloat16 *in, const __nv_bfloat16 *dy, float *part,
              float *gw, float *gb, cudaStream_t st) {
  if (cin == 32 && cout == 32)
    dw_launch<32, 32>(g, in, dy, part, gw, st);
  else if (cin == 16 && cout == 32)
    dw_launch<16, 32>(g, in, dy, part, gw, st);
  else if (cin == 32 && cout == 16)
    dw_launch<32, 16>(g, in, dy, part, gw, st);
  else
    dw_launch<16, 16>(g, in, dy, part, gw, st);
  bias_part_kernel<<<BIAS_CTAS, 128, 0, st>>>(g.voxels(), cout, dy, part);
  bias_reduce_kernel<<<1, 32, 0, st>>>(BIAS_CTAS, cout, part, gb);
}

void flip_weights(int cin, int cout, const __nv_bfloat16 *w, __nv_bfloat16 *wt, cudaStream_t st) {
  flip_kernel<<<grid_for(27 * cin * cout), 256, 0, st>>>(cin, cout, w, wt);
}

void to_bf16(int64_t n, const float *src, __nv_bfloat16 *dst, cudaStream_t st) {
  to_bf16_kernel<<<grid_for(n), 256, 0, st>>>(n, src, dst);
}

void pool(const Grid &gf, const Grid &gc, const __nv_bfloat16 *fine, __nv_bfloat16 *coarse, cudaStream_t st) {
  pool_kernel<<<grid_for(gc.voxels() * 16), 256, 0, st>>>(gf, gc, fine, coarse);
}
void up_add(const Grid &gf, const Grid &gc, const __nv_bfloat16 *coarse, const __nv_bfloat16 *skip,
            __nv_bfloat16 *fine, cudaStream_t st) {
  up_add_kernel<<<grid_for(gf.voxels() * 16), 256, 0, st>>>(gf, gc, coarse, skip, fine);
}
void up_adjoint(const Grid &gf, const Grid &gc, const __nv_bfloat16 *dfine, const __nv_bfloat16 *mask,
                __nv_bfloat16 *dcoarse, cudaStream_t st) {
  up_adjoint_kernel<<<grid_for(gc.voxels() * 16), 256, 0, st>>>(gf, gc, dfine, mask, dcoarse);
}
void pool_adjoint(const Grid &gf, const Grid &gc, const __nv_bfloat16 *dcoarse, const __nv_bfloat16 *dskip,
                  const __nv_bfloat16 *mask, __nv_bfloat16 *dfine, cudaStream_t st) {
  pool_adjoint_kernel<<<grid_for(gf.voxels() * 16), 256, 0, st>>>(gf, gc, dcoarse, dskip, mask, dfine);
}

void scatter_input(const Grid &g, const int64_t *eq, const double *r, const float *feat, const double *scale,
                   __nv_bfloat16 *x, cudaStream_t st) {
  scatter_input_kernel<<<grid_for(g.voxels() * CIO), 256, 0, st>>>(g, eq, r, feat, scale, x);
}
void gather_output(const Grid &g, const int64_t *eq, const __nv_bfloat16 *y, const double *scale, double *z,
                   cudaStream_t st) {
  gather_output_kernel<<<grid_for(g.voxels() * 3), 256, 0, st>>>(g, eq, y, scale, z);
}
void scatter_grad(const Grid &g, const int64_t *eq, const double *dz, const double *scale, __nv_bfloat16 *dy,
                  cudaStream_t st) {
  scatter_grad_kernel<<<grid_for(g.voxels() * CIO), 256, 0, st>>>(g, eq, dz, scale, dy);
}

void adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
          cudaStream_t st) {
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  adam_kernel<<<grid_for(n), 256, 0, st>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
}

void dots(int64_t n, int pairs, const double *const *a, const double *const *b, double *partial, double *out,
          cudaStream_t st) {
  PairPtrs pp{};
  for (int k = 0; k < pairs && k < MAX_PAIRS; ++k) pp.a[k] = a[k], pp.b[k] = b[k];
  dot_part_kernel<<<DOT_CTAS, 256, 0, st>>>(n, pairs, pp, partial);
  dot_final_kernel<<<1, 256, 0, st>>>(DOT_CTAS, pairs, partial, out);
}

void axpy_dev(int64_t n, const double *alpha, double sign, const double *x, double *y, cudaStream_t st) {
  axpy_dev_kernel<<<grid_for(n), 256, 0, st>>>(n, alpha, sign, x, y);
}

void fcg_direction(int64_t n, int m, const double *z, const double *const *pj, const int *slot, const double *num,
                   const double *den, double *p, cudaStream_t st) {
  DirPtrs dp{};
  for (int j = 0; j < m && j < MAX_PAIRS; ++j) dp.p[j] = pj[j], dp.slot[j] = slot[j];
  fcg_direction_kernel<<<grid_for(n), 256, 0, st>>>(n, m, z, dp, num, den, p);
}

// alpha = s[0] / s[1] (p.r / p.q; 0 when p.q is 0), kept: *den = s[1]; x += alpha p; r -= alpha q
__global__ void fcg_update_kernel(int64_t n, const double *__restrict__ s, double *__restrict__ den,
                                  const double *__restrict__ p, const double *__restrict__ q, double *__restrict__ x,
                                  double *__restrict__ r) {
  const double alpha = s[1] != 0.0 ? s[0] / s[1] : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *den = s[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    r[i] -= alpha * q[i];
  }
}
void fcg_update(int64_t n, const double *s, double *den, const double *p, const double *q, double *x, double *r,
                cudaStream_t st) {
  fcg_update_kernel<<<grid_for(n), 256, 0, st>>>(n, s, den, p, q, x, r);
}

void input_scales(int64_t n, const double *nrm2, double kref, double *s, cudaStream_t st) {
  input_scales_kernel<<<1, 1, 0, st>>>(n, nrm2, kref, s);
}

}  // namespace unet
}  // namespace fc
