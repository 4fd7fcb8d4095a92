// Kernels of the learned surrogate (a Fourier neural operator over the design
// density): a batched BF16 tensor-core GEMM with FP32 accumulation and fused
// epilogues, the per-mode complex channel mixing of the spectral layers, and the
// small elementwise kernels of training (GELU backward, pixel mean, Adam).
// No counterpart in the reference, which has no learned surrogate.
//
// GEMM: C[b] = epilogue(alpha * op(A[b]) @ op(B[b])). Block tiles of BM x BN x 32
// are staged through registers into padded shared memory with the reduction dim
// (K) contiguous whatever the operands' layouts (80-byte rows keep ldmatrix free
// of bank conflicts), double buffered, and multiplied by warps with
// mma.sync.m16n8k16 (bf16 inputs, f32 accumulators). The epilogue adds an f32 (or
// bf16) term, row/column biases, applies GELU, and stores f32 and/or bf16, or
// accumulates atomically (batch-reduced or split-K weight gradients). Where the
// shapes allow, bz_gemm_bf16 runs tcgen05/TMEM kernels instead: the large DFT GEMMs
// (TMA-fed, 128 x 256 tiles), the 1x1 channel mixing (pixel-contiguous activations
// as an MN-major TMA operand) and its weight gradients (both operands K-major,
// reduced over pixels and designs); each is described below. The mma.sync kernel
// remains for the shapes they do not take (the 3-channel lift layer, the pooled head).
#include <cuda.h>
#include <cuda_bf16.h>

#include <mutex>

#include "bz_internal.cuh"

namespace bz {
namespace {

typedef __nv_bfloat16 bf16;
constexpr int GBK = 32;
constexpr int GPAD = 8;
constexpr int GLD = GBK + GPAD;  // smem row length in bf16 elements (80 bytes)

struct GemmP {
  int M, N, K, batch, splitk, act, ta, tb, atomic;
  const bf16* A;
  long long lda, sa;
  const bf16* B;
  long long ldb, sb;
  float alpha;
  const float* cadd;
  long long ldadd, sadd;
  const float* bias_m;
  const float* bias_n;
  float* outf;
  bf16* outh;
  long long ldc, sc;
  bf16* pre;
  long long ldpre, spre;
  const bf16* cadd_h;  // the added term in bf16 instead of f32 (same strides), or null
  int wait_limit;  // polls of a bounded mbarrier wait before it gives up (tcgen05 kernel)
  int withhold;    // 1: the tcgen05 kernel issues no MMA for its first K slice (timeout self-test)
};

__device__ __forceinline__ float gelu_f(float v) {
  // tanh form of GELU
  const float u = 0.7978845608028654f * (v + 0.044715f * v * v * v);
  return 0.5f * v * (1.0f + tanhf(u));
}

// GELU (tanh form) for results stored only as bf16: the PTX tanh.approx.f32 instruction
// (relative error about 2^-11) is below the 2^-9 rounding of the bf16 store.
__device__ __forceinline__ float gelu_bf16out(float v) {
  const float u = 0.7978845608028654f * (v + 0.044715f * v * v * v);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * v * (1.0f + t);
}

__device__ __forceinline__ float gelu_grad(float v) {
  const float u = 0.7978845608028654f * (v + 0.044715f * v * v * v);
  const float t = tanhf(u);
  const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * v * v);
  return 0.5f * (1.0f + t) + 0.5f * v * (1.0f - t * t) * du;
}

// 8 consecutive bf16 from p (elements idx .. idx+7 of a line with `lim` valid ones);
// zero beyond the line or when !ok.
__device__ __forceinline__ uint4 load8(const bf16* p, long long idx, long long lim, bool ok) {
  uint4 r = make_uint4(0u, 0u, 0u, 0u);
  if (!ok || idx >= lim) return r;
  const bf16* q = p + idx;
  if (idx + 8 <= lim && ((reinterpret_cast<uintptr_t>(q) & 15u) == 0u)) return __ldg(reinterpret_cast<const uint4*>(q));
  unsigned short* h = reinterpret_cast<unsigned short*>(&r);
  const unsigned short* s = reinterpret_cast<const unsigned short*>(q);
  const int n = (int)min(8LL, lim - idx);
  for (int i = 0; i < n; ++i) h[i] = s[i];
  return r;
}

__device__ __forceinline__ void ldsm_x4(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, const bf16* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int BM, int BN, int WM, int WN>
__global__ void __launch_bounds__(32 * WM * WN) gemm_bf16_kernel(GemmP p) {
  constexpr int NT_ = 32 * WM * WN;
  constexpr int TM = BM / WM, TN = BN / WN;  // warp tile
  constexpr int MT = TM / 16, NT = TN / 8;
  static_assert(NT % 2 == 0 && MT >= 1, "warp tile");
  constexpr int CA = (BM * GBK / 8 + NT_ - 1) / NT_;  // 8-element chunks per thread
  constexpr int CB = (BN * GBK / 8 + NT_ - 1) / NT_;
  __shared__ __align__(16) bf16 As[2][BM][GLD];
  __shared__ __align__(16) bf16 Bs[2][BN][GLD];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp / WN) * TM, wn0 = (warp % WN) * TN;
  const int bz = blockIdx.z / p.splitk, ks = blockIdx.z % p.splitk;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const bf16* A = p.A + (long long)bz * p.sa;
  const bf16* B = p.B + (long long)bz * p.sb;
  const int ktiles = (p.K + GBK - 1) / GBK;
  const int kper = (ktiles + p.splitk - 1) / p.splitk;
  const int kt0 = ks * kper, kt1 = min(ktiles, kt0 + kper);

  uint4 ra[CA], rb[CB];
  auto gload = [&](int kt) {
    const int k0 = kt * GBK;
#pragma unroll
    for (int c = 0; c < CA; ++c) {
      const int ch = tid + c * NT_;
      if (ch >= BM * GBK / 8) break;
      if (!p.ta) {  // A[m][k], k contiguous
        const int r = ch / (GBK / 8), kc = (ch % (GBK / 8)) * 8;
        const int m = m0 + r;
        ra[c] = load8(A + (long long)min(m, p.M - 1) * p.lda, k0 + kc, p.K, m < p.M);
      } else {  // A stored [k][m], m contiguous
        const int k = ch / (BM / 8), mc = (ch % (BM / 8)) * 8;
        ra[c] = load8(A + (long long)min(k0 + k, p.K - 1) * p.lda, m0 + mc, p.M, k0 + k < p.K);
      }
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      const int ch = tid + c * NT_;
      if (ch >= BN * GBK / 8) break;
      if (p.tb) {  // B stored [n][k], k contiguous
        const int r = ch / (GBK / 8), kc = (ch % (GBK / 8)) * 8;
        const int n = n0 + r;
        rb[c] = load8(B + (long long)min(n, p.N - 1) * p.ldb, k0 + kc, p.K, n < p.N);
      } else {  // B[k][n], n contiguous
        const int k = ch / (BN / 8), nc = (ch % (BN / 8)) * 8;
        rb[c] = load8(B + (long long)min(k0 + k, p.K - 1) * p.ldb, n0 + nc, p.N, k0 + k < p.K);
      }
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int c = 0; c < CA; ++c) {
      const int ch = tid + c * NT_;
      if (ch >= BM * GBK / 8) break;
      if (!p.ta) {
        const int r = ch / (GBK / 8), kc = (ch % (GBK / 8)) * 8;
        *reinterpret_cast<uint4*>(&As[buf][r][kc]) = ra[c];
      } else {
        const int k = ch / (BM / 8), mc = (ch % (BM / 8)) * 8;
        const bf16* h = reinterpret_cast<const bf16*>(&ra[c]);
#pragma unroll
        for (int i = 0; i < 8; ++i) As[buf][mc + i][k] = h[i];
      }
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      const int ch = tid + c * NT_;
      if (ch >= BN * GBK / 8) break;
      if (p.tb) {
        const int r = ch / (GBK / 8), kc = (ch % (GBK / 8)) * 8;
        *reinterpret_cast<uint4*>(&Bs[buf][r][kc]) = rb[c];
      } else {
        const int k = ch / (BN / 8), nc = (ch % (BN / 8)) * 8;
        const bf16* h = reinterpret_cast<const bf16*>(&rb[c]);
#pragma unroll
        for (int i = 0; i < 8; ++i) Bs[buf][nc + i][k] = h[i];
      }
    }
  };

  float acc[MT][NT][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  if (kt0 < kt1) {
    gload(kt0);
    sstore(0);
    __syncthreads();
    for (int kt = kt0; kt < kt1; ++kt) {
      const int buf = (kt - kt0) & 1;
      if (kt + 1 < kt1) gload(kt + 1);
#pragma unroll
      for (int kk = 0; kk < GBK; kk += 16) {
        unsigned af[MT][4], bfr[NT][2];
#pragma unroll
        for (int i = 0; i < MT; ++i)
          ldsm_x4(af[i][0], af[i][1], af[i][2], af[i][3], &As[buf][wm0 + i * 16 + (lane & 15)][kk + (lane >> 4) * 8]);
#pragma unroll
        for (int j = 0; j < NT; j += 2)
          ldsm_x4(bfr[j][0], bfr[j][1], bfr[j + 1][0], bfr[j + 1][1],
                  &Bs[buf][wn0 + j * 8 + (lane & 7) + ((lane >> 4) << 3)][kk + ((lane >> 3) & 1) * 8]);
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], af[i], bfr[j][0], bfr[j][1]);
      }
      if (kt + 1 < kt1) sstore(buf ^ 1);
      __syncthreads();
    }
  }

  // epilogue: each thread holds pairs of adjacent columns (e, e+1); pairs go through
  // 8-byte f32 and 4-byte bf16x2 accesses when both columns exist and the row offsets
  // are even, single elements otherwise
  const bool even = ((p.ldc | p.sc | p.ldadd | p.sadd | p.ldpre | p.spre) & 1) == 0 &&
                    ((reinterpret_cast<uintptr_t>(p.cadd) | reinterpret_cast<uintptr_t>(p.outf)) & 7u) == 0 &&
                    ((reinterpret_cast<uintptr_t>(p.outh) | reinterpret_cast<uintptr_t>(p.pre)) & 3u) == 0;
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm0 + i * 16 + (lane >> 2) + h * 8;
        const int n = n0 + wn0 + j * 8 + (lane & 3) * 2;
        if (m >= p.M || n >= p.N) continue;
        float v[2] = {p.alpha * acc[i][j][2 * h], p.alpha * acc[i][j][2 * h + 1]};
        const bool pair = even && n + 1 < p.N && !p.atomic;
        const int cnt = n + 1 < p.N ? 2 : 1;
        if (p.cadd) {
          const float* q = p.cadd + (long long)bz * p.sadd + (long long)m * p.ldadd + n;
          if (pair) {
            const float2 a = *reinterpret_cast<const float2*>(q);
            v[0] += a.x;
            v[1] += a.y;
          } else {
            for (int e = 0; e < cnt; ++e) v[e] += q[e];
          }
        } else if (p.cadd_h) {
          const bf16* q = p.cadd_h + (long long)bz * p.sadd + (long long)m * p.ldadd + n;
          for (int e = 0; e < cnt; ++e) v[e] += __bfloat162float(q[e]);
        }
        for (int e = 0; e < cnt; ++e) {
          if (p.bias_m) v[e] += p.bias_m[m];
          if (p.bias_n) v[e] += p.bias_n[n + e];
        }
        if (p.pre) {
          bf16* q = p.pre + (long long)bz * p.spre + (long long)m * p.ldpre + n;
          if (pair) *reinterpret_cast<__nv_bfloat162*>(q) = __floats2bfloat162_rn(v[0], v[1]);
          else for (int e = 0; e < cnt; ++e) q[e] = __float2bfloat16_rn(v[e]);
        }
        if (p.act == 1) {
          v[0] = gelu_f(v[0]);
          v[1] = gelu_f(v[1]);
        }
        const long long o = (long long)bz * p.sc + (long long)m * p.ldc + n;
        if (p.outf) {
          if (p.atomic) {
            for (int e = 0; e < cnt; ++e) atomicAdd(p.outf + o + e, v[e]);
          } else if (pair) {
            *reinterpret_cast<float2*>(p.outf + o) = make_float2(v[0], v[1]);
          } else {
            for (int e = 0; e < cnt; ++e) p.outf[o + e] = v[e];
          }
        }
        if (p.outh) {
          if (pair) *reinterpret_cast<__nv_bfloat162*>(p.outh + o) = __floats2bfloat162_rn(v[0], v[1]);
          else for (int e = 0; e < cnt; ++e) p.outh[o + e] = __float2bfloat16_rn(v[e]);
        }
      }
}

template <int BM, int BN, int WM, int WN>
int launch_gemm(const GemmP& p, cudaStream_t st) {
  dim3 grid((unsigned)ceil_div(p.N, BN), (unsigned)ceil_div(p.M, BM), (unsigned)(p.batch * p.splitk));
  gemm_bf16_kernel<BM, BN, WM, WN><<<grid, 32 * WM * WN, 0, st>>>(p);
  return check_launch("bz_gemm_bf16");
}


// ---- tcgen05 path: A row-major (K contiguous) x B stored [N][K] (K contiguous) ------
// One CTA of 128 threads computes a 128 x 256 tile into 256 TMEM columns (f32). Per
// 64-wide K slice, the threads stage A (128 x 64) and B (256 x 64) in shared memory in
// the no-swizzle K-major core-matrix layout (8 rows x 16 bytes per core matrix; 8-row
// groups 128 bytes apart, K chunks LBO apart, LBO padded by 16 bytes so that the
// 16-byte stores of a warp spread over all banks); one thread issues four
// tcgen05.mma (K = 16 each, kind::f16 with bf16 A and B) and commits them to the
// stage's mbarrier. Two stages: the next slice's global loads overlap the MMAs. The
// epilogue reads the accumulators with tcgen05.ld (warp w owns rows 32w..32w+31).
// Every mbarrier wait is bounded; a timeout raises g_tc_error and the CTA frees its
// TMEM and returns.
namespace tc {
constexpr int BM = 128, BN = 256, BK = 64, THREADS = 128;
constexpr int LBO_A = (BM / 8) * 128 + 16, LBO_B = (BN / 8) * 128 + 16;
constexpr int A_BYTES = 8 * LBO_A, B_BYTES = 8 * LBO_B;  // 8 K chunks of 8 elements
constexpr int STAGE = A_BYTES + B_BYTES;
constexpr int SMEM = 2 * STAGE + 64;
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);  // f32 accum, bf16 A/B, K-major, M=128, N=256
constexpr int WAIT_LIMIT = 1 << 22;
}  // namespace tc

__device__ int g_tc_error = 0;

__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
  return d;
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, int limit = tc::WAIT_LIMIT) {
  for (int i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__global__ void __launch_bounds__(tc::THREADS) gemm_tc_kernel(GemmP p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int bz = blockIdx.z / p.splitk, ks = blockIdx.z % p.splitk;
  const int m0 = blockIdx.y * tc::BM, n0 = blockIdx.x * tc::BN;
  const bf16* A = p.A + (long long)bz * p.sa;
  const bf16* B = p.B + (long long)bz * p.sb;
  const int ktiles = (p.K + tc::BK - 1) / tc::BK;
  const int kper = (ktiles + p.splitk - 1) / p.splitk;
  const int kt0 = ks * kper, kt1 = min(ktiles, kt0 + kper);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * tc::STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 2 * tc::STAGE + 16);
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t mb0 = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar[0]));

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot))),
                 "r"(tc::BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0 + 8));
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t taddr = *tmem_slot;

  // global -> registers: A 8 chunks and B 16 chunks of 16 bytes per thread
  uint4 ra[8], rb[16];
  auto gload = [&](int kt) {
    const int k0 = kt * tc::BK;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = tid + i * tc::THREADS, r = c >> 3, j = c & 7;
      const int m = m0 + r;
      ra[i] = load8(A + (long long)min(m, p.M - 1) * p.lda, k0 + j * 8, p.K, m < p.M);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int c = tid + i * tc::THREADS, r = c >> 3, j = c & 7;
      const int n = n0 + r;
      rb[i] = load8(B + (long long)min(n, p.N - 1) * p.ldb, k0 + j * 8, p.K, n < p.N);
    }
  };
  auto sstore = [&](int s) {
    unsigned char* st = smem + s * tc::STAGE;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = tid + i * tc::THREADS, r = c >> 3, j = c & 7;
      *reinterpret_cast<uint4*>(st + j * tc::LBO_A + (r >> 3) * 128 + (r & 7) * 16) = ra[i];
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int c = tid + i * tc::THREADS, r = c >> 3, j = c & 7;
      *reinterpret_cast<uint4*>(st + tc::A_BYTES + j * tc::LBO_B + (r >> 3) * 128 + (r & 7) * 16) = rb[i];
    }
  };

  uint32_t phase[2] = {0u, 0u};
  bool ok = true;
  int last = -1;
  if (kt0 < kt1) {
    gload(kt0);
    sstore(0);
    for (int kt = kt0; kt < kt1 && ok; ++kt) {
      const int s = (kt - kt0) & 1;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (tid == 0 && !(p.withhold && kt == kt0)) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t a0 = sbase + s * tc::STAGE, b0 = a0 + tc::A_BYTES;
#pragma unroll
        for (int kk = 0; kk < tc::BK / 16; ++kk) {
          const uint64_t da = tc_sdesc(a0 + kk * 2 * tc::LBO_A, tc::LBO_A, 128);
          const uint64_t db = tc_sdesc(b0 + kk * 2 * tc::LBO_B, tc::LBO_B, 128);
          const uint32_t acc = (kt > kt0 || kk > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
              :
              : "r"(taddr), "l"(da), "l"(db), "r"(tc::IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            mb0 + 8 * s));
      }
      last = s;
      if (kt + 1 < kt1) {
        gload(kt + 1);
        const int s2 = s ^ 1;
        if (kt > kt0) {  // the MMAs of the previous slice read stage s2
          ok = tc_wait(mb0 + 8 * s2, phase[s2], p.wait_limit);
          phase[s2] ^= 1u;
        }
        if (ok) sstore(s2);
      }
      ok = __syncthreads_and(ok);
    }
    if (ok) {
      ok = tc_wait(mb0 + 8 * last, phase[last], p.wait_limit);
    } else if (!(p.withhold && last == 0 && kt1 - kt0 == 1)) {
      tc_wait(mb0 + 8 * last, phase[last], p.wait_limit);  // let issued MMAs drain before the TMEM goes
    }
    if (!ok && tid == 0) atomicExch(&g_tc_error, 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  // epilogue: thread (warp w, lane l) owns row 32w + l of the tile
  const int m = m0 + warp * 32 + lane;
  if (__syncthreads_and(ok)) {
    for (int c0 = 0; c0 < tc::BN; c0 += 8) {
      uint32_t v[8];
      if (kt0 < kt1) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
            : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = 0u;
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int n = n0 + c0 + e;
        if (m >= p.M || n >= p.N) continue;
        float x = p.alpha * __uint_as_float(v[e]);
        if (p.cadd) x += p.cadd[(long long)bz * p.sadd + (long long)m * p.ldadd + n];
        else if (p.cadd_h) x += __bfloat162float(p.cadd_h[(long long)bz * p.sadd + (long long)m * p.ldadd + n]);
        if (p.bias_m) x += p.bias_m[m];
        if (p.bias_n) x += p.bias_n[n];
        if (p.pre) p.pre[(long long)bz * p.spre + (long long)m * p.ldpre + n] = __float2bfloat16_rn(x);
        if (p.act == 1) x = gelu_f(x);
        const long long o = (long long)bz * p.sc + (long long)m * p.ldc + n;
        if (p.outf) {
          if (p.atomic) atomicAdd(p.outf + o, x); else p.outf[o] = x;
        }
        if (p.outh) p.outh[o] = __float2bfloat16_rn(x);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(tc::BN));
}

int launch_gemm_tc(const GemmP& p, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM) != cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_gemm_bf16: cannot configure the tcgen05 kernel's shared memory");
    configured = true;
  }
  dim3 grid((unsigned)ceil_div(p.N, tc::BN), (unsigned)ceil_div(p.M, tc::BM), (unsigned)(p.batch * p.splitk));
  gemm_tc_kernel<<<grid, tc::THREADS, tc::SMEM, st>>>(p);
  return check_launch("bz_gemm_bf16");
}


// ---- tcgen05 + TMA path (batch 1): one control thread, four-stage pipeline --------
// Operand stages are filled by TMA tiled copies with 128-byte swizzling (2D tensor
// maps over the row-major K-contiguous A and B, box 64 elements x 128 or 256 rows: one
// copy per operand per stage), which is the K-major SWIZZLE_128B layout of the MMA
// descriptors (8-row atoms of 128-byte rows, atoms 1024 bytes apart; the K step of 16
// elements advances the start address by 32 bytes inside the atom). Thread 0 waits for
// a stage's copies (mbarrier complete_tx), issues its four MMAs, commits them to the
// stage's "empty" barrier, and refills the previous stage once its MMAs are done, so
// the tensor pipe always has queued work. Four 48 KB stages (192 KB, one CTA per SM)
// keep three tiles of loads in flight behind the MMAs: with two, the next tile's load
// latency (about a microsecond) outlasted a tile's MMAs and the tensor pipe idled.
// Bounded waits as above.
namespace tma {
constexpr int S = 4, BK = 64;
constexpr int A_ST = tc::BM * BK * 2, B_ST = tc::BN * BK * 2, STAGE = A_ST + B_ST;
constexpr int SMEM = S * STAGE + 1024 + 128;  // + alignment slack + barriers
}  // namespace tma

// K-major SWIZZLE_128B operand descriptor: start address, leading offset unused (1),
// stride 1024 bytes between 8-row atoms, sm_100 version bits, layout type 2.
__device__ __forceinline__ uint64_t tc_sdesc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

__global__ void __launch_bounds__(tc::THREADS) gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB, GemmP p) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ks = blockIdx.z;
  const int m0 = blockIdx.y * tc::BM, n0 = blockIdx.x * tc::BN;
  const int ktiles = (p.K + tma::BK - 1) / tma::BK;
  const int kper = (ktiles + p.splitk - 1) / p.splitk;
  const int kt0 = ks * kper, kt1 = min(ktiles, kt0 + kper);
  const int nt = max(0, kt1 - kt0);
  unsigned char* bar = smem + tma::S * tma::STAGE;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 8 * (2 * tma::S + 1));
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t full0 = static_cast<uint32_t>(__cvta_generic_to_shared(bar));
  const uint32_t empty0 = full0 + 8 * tma::S, done = full0 + 16 * tma::S;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot))),
                 "r"(tc::BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < 2 * tma::S + 1; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(full0 + 8 * i));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t taddr = *tmem_slot;

  int ok = 1;
  if (tid == 0 && nt > 0) {
    auto issue = [&](int t) {  // tile kt0 + t into stage t % S
      const int s = t % tma::S, k0 = (kt0 + t) * tma::BK;
      const uint32_t st = sbase + s * tma::STAGE, fb = full0 + 8 * s;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(tma::STAGE) : "memory");
      tma_load_2d(st, &tmA, k0, m0, fb);
      tma_load_2d(st + tma::A_ST, &tmB, k0, n0, fb);
    };
    int issued = 0, consumed = 0;
    for (; issued < min(tma::S, nt); ++issued) issue(issued);
    for (int it = 0; it < nt; ++it) {
      const int s = it % tma::S;
      if (!tc_wait(full0 + 8 * s, (uint32_t)((it / tma::S) & 1))) {
        ok = 0;
        break;
      }
      consumed = it + 1;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t a0 = sbase + s * tma::STAGE, b0 = a0 + tma::A_ST;
#pragma unroll
      for (int kk = 0; kk < tma::BK / 16; ++kk) {
        const uint64_t da = tc_sdesc_sw128(a0 + kk * 32);
        const uint64_t db = tc_sdesc_sw128(b0 + kk * 32);
        const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            :
            : "r"(taddr), "l"(da), "l"(db), "r"(tc::IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          empty0 + 8 * s));
      if (it >= 1 && issued < nt) {  // refill the previous stage once its MMAs are done
        const int sp = (it - 1) % tma::S;
        if (!tc_wait(empty0 + 8 * sp, (uint32_t)(((it - 1) / tma::S) & 1))) {
          ok = 0;
          break;
        }
        issue(issued++);
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(done));
    for (int t = consumed; t < issued; ++t)  // copies still in flight after a failure
      tc_wait(full0 + 8 * (t % tma::S), (uint32_t)((t / tma::S) & 1));
  }
  ok = __syncthreads_and(ok);
  if (nt > 0) {
    if (!tc_wait(done, 0u)) ok = 0;
  }
  ok = __syncthreads_and(ok);
  if (!ok && tid == 0) atomicExch(&g_tc_error, 1);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const int m = m0 + warp * 32 + lane;
  // plain f32 output (no epilogue terms): two 16-byte stores per 8 columns
  const bool plain = p.outf && !p.atomic && !p.outh && !p.cadd && !p.cadd_h && !p.bias_m && !p.bias_n && !p.pre && p.act == 0 &&
                     (p.ldc & 3) == 0 && ((reinterpret_cast<uintptr_t>(p.outf) & 15u) == 0u);
  // plain bf16 output: one 16-byte store per 8 columns
  const bool plain_h = p.outh && !p.outf && !p.atomic && !p.cadd && !p.cadd_h && !p.bias_m && !p.bias_n && !p.pre &&
                       p.act == 0 && (p.ldc & 7) == 0 && ((reinterpret_cast<uintptr_t>(p.outh) & 15u) == 0u);
  if (ok) {
    for (int c0 = 0; c0 < tc::BN; c0 += 8) {
      uint32_t v[8];
      if (nt > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
            : "r"(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = 0u;
      }
      if (plain && m < p.M && n0 + c0 + 8 <= p.N) {
        float4* q = reinterpret_cast<float4*>(p.outf + (long long)m * p.ldc + n0 + c0);
        q[0] = make_float4(p.alpha * __uint_as_float(v[0]), p.alpha * __uint_as_float(v[1]),
                           p.alpha * __uint_as_float(v[2]), p.alpha * __uint_as_float(v[3]));
        q[1] = make_float4(p.alpha * __uint_as_float(v[4]), p.alpha * __uint_as_float(v[5]),
                           p.alpha * __uint_as_float(v[6]), p.alpha * __uint_as_float(v[7]));
      } else if (plain_h && m < p.M && n0 + c0 + 8 <= p.N) {
        uint4 w;
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&w);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          h[e] = __floats2bfloat162_rn(p.alpha * __uint_as_float(v[2 * e]), p.alpha * __uint_as_float(v[2 * e + 1]));
        *reinterpret_cast<uint4*>(p.outh + (long long)m * p.ldc + n0 + c0) = w;
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int n = n0 + c0 + e;
          if (m >= p.M || n >= p.N) continue;
          float x = p.alpha * __uint_as_float(v[e]);
          if (p.cadd) x += p.cadd[(long long)m * p.ldadd + n];
          else if (p.cadd_h) x += __bfloat162float(p.cadd_h[(long long)m * p.ldadd + n]);
          if (p.bias_m) x += p.bias_m[m];
          if (p.bias_n) x += p.bias_n[n];
          if (p.pre) p.pre[(long long)m * p.ldpre + n] = __float2bfloat16_rn(x);
          if (p.act == 1) x = gelu_f(x);
          const long long o = (long long)m * p.ldc + n;
          if (p.outf) {
            if (p.atomic) atomicAdd(p.outf + o, x); else p.outf[o] = x;
          }
          if (p.outh) p.outh[o] = __float2bfloat16_rn(x);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(tc::BN));
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

// 2D map over a row-major bf16 matrix of `rows` x `cols` (cols contiguous, ld elements
// per row), box 64 columns (128 bytes, the swizzle span) x box_rows rows, 128-byte
// swizzle; out-of-range elements read as zero.
bool make_map(CUtensorMap* map, const bf16* base, long long rows, long long cols, long long ld, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t stride[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)tma::BK, (cuuint32_t)box_rows};
  const cuuint32_t estride[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dim, stride, box, estride,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 1: launched; 0: not applicable here (caller uses another kernel); <0: error status.
int launch_gemm_tma(const GemmP& p, cudaStream_t st) {
  if (p.batch != 1) return 0;
  alignas(64) CUtensorMap ma, mb;
  if (!make_map(&ma, p.A, p.M, p.K, p.lda, tc::BM) || !make_map(&mb, p.B, p.N, p.K, p.ldb, tc::BN)) return 0;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(gemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tma::SMEM) != cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_gemm_bf16: cannot configure the TMA kernel's shared memory");
    configured = true;
  }
  dim3 grid((unsigned)ceil_div(p.N, tc::BN), (unsigned)ceil_div(p.M, tc::BM), (unsigned)p.splitk);
  gemm_tma_kernel<<<grid, tc::THREADS, tma::SMEM, st>>>(ma, mb, p);
  const int rc = check_launch("bz_gemm_bf16");
  return rc == BZ_OK ? 1 : rc;
}

bool tc_eligible(const GemmP& p) {
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0u; };
  return !p.ta && p.tb && p.M >= 128 && p.N >= 256 && p.K >= 64 && p.lda % 8 == 0 && p.ldb % 8 == 0 &&
         p.sa % 8 == 0 && p.sb % 8 == 0 && al(p.A) && al(p.B);
}

// ---- tcgen05 channel mixing: C[b] = epilogue(W (M x K) @ X[b] (K x N)), X pixel-contiguous ----
// The surrogate's 1x1 layers: X[b] is [K][N] with the N pixels contiguous and W a small
// weight (M, K in {32, 64}) shared by the batch. Computed transposed, D[b] (N x M) =
// X[b]^T W^T: the pixels are the MMA's M (128 per tile), the output channels its N.
// X is therefore an MN-major A operand. TMA stages it with 128-byte swizzling as two
// 64-pixel boxes of K rows per tile; that is the MN-major SWIZZLE_128B layout of the
// descriptor (8-row atoms of 128-byte rows along K, atoms SBO = 1024 bytes apart, the
// second 64-pixel block LBO = 128 K bytes after the first; a K step of 16 moves the
// start address by two atoms). W^T is the K-major B operand, written once per CTA by
// the threads in the no-swizzle core-matrix layout. A persistent CTA of 128 threads
// walks tiles (design b, 128 pixels) with a four-stage TMA ring and two TMEM
// accumulators of M columns: while the four warps run tile j's epilogue, thread 0 has
// already issued tile j+1's K/16 MMAs into the other accumulator. Each warp first loads
// its 32 pixels' f32 term (independent of the MMAs), then waits for tile j's commit,
// reads its rows with tcgen05.ld and applies the epilogue (f32 term, biases,
// pre-activation, GELU), every load and store coalesced along the pixels. Memory-bound
// (K = 32: 64 bytes read and 64-192 bytes written per pixel), so the grid is sized for
// as many CTAs per SM as registers, shared memory and TMEM allow, and their epilogues
// keep loads in flight. Bounded waits as in the GEMMs above.
namespace mix {
constexpr int S = 4, TP = 128, THREADS = 128;
}

// MN-major SWIZZLE_128B operand descriptor: LBO = distance between the 64-element MN
// blocks, SBO = 1024 bytes between 8-row K atoms, sm_100 version bits, layout type 2.
__device__ __forceinline__ uint64_t tc_sdesc_sw128_mn(uint32_t saddr, uint32_t lbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int KC, int MC>
struct MixCfg {
  static constexpr int A_ST = 2 * KC * 128;  // two 64-pixel boxes of KC rows (bytes)
  static constexpr int W_OFF = mix::S * A_ST;
  static constexpr int LBO_W = (MC / 8) * 128;
  static constexpr int BAR_OFF = W_OFF + MC * KC * 2;
  static constexpr int SMEM = BAR_OFF + 8 * (mix::S + 3) + 1024;  // + alignment slack
  static constexpr int NCOL = MC < 32 ? 32 : MC;                   // columns of one accumulator
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | ((uint32_t)(MC >> 3) << 17) |
                                    ((uint32_t)(mix::TP >> 4) << 24);  // f32 += bf16 x bf16, A MN-major
};

template <int KC, int MC>
__global__ void __launch_bounds__(mix::THREADS) mix_tc_kernel(const __grid_constant__ CUtensorMap tmX, GemmP p,
                                                             int n_tiles, int tiles_n) {
  using C = MixCfg<KC, MC>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* bar = smem + C::BAR_OFF;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 8 * (mix::S + 2));
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  // barriers: full[S] (TMA), mdone[2] (MMAs of the accumulator pair)
  const uint32_t full0 = static_cast<uint32_t>(__cvta_generic_to_shared(bar)), mdone0 = full0 + 8 * mix::S;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot))),
                 "r"(2 * C::NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < mix::S + 2; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(full0 + 8 * i));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // W^T (rows = output channels m, K contiguous) in the no-swizzle K-major layout
  for (int i = tid; i < MC * KC; i += mix::THREADS) {
    const int m = i / KC, k = i - (i / KC) * KC;
    const bf16 w = p.ta ? p.A[(long long)k * p.lda + m] : p.A[(long long)m * p.lda + k];
    *reinterpret_cast<bf16*>(smem + C::W_OFF + (k >> 3) * C::LBO_W + (m >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2) = w;
  }
  __shared__ float s_bias[MC];
  for (int i = tid; i < MC; i += mix::THREADS) s_bias[i] = p.bias_m ? p.bias_m[i] : 0.f;
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t taddr = *tmem_slot;

  const int n_my = (n_tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  auto issue = [&](int j) {  // this CTA's tile j into stage j % S
    const int t = (int)blockIdx.x + j * (int)gridDim.x;
    const int b = t / tiles_n, n0 = (t - b * tiles_n) * mix::TP;
    const uint32_t st = sbase + (j % mix::S) * C::A_ST, fb = full0 + 8 * (j % mix::S);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(C::A_ST) : "memory");
    tma_load_2d(st, &tmX, n0, b * KC, fb);
    tma_load_2d(st + KC * 128, &tmX, n0 + 64, b * KC, fb);
  };
  // tile j's MMAs into accumulator j & 1 (thread 0); false when its operands never landed
  auto mma = [&](int j) -> bool {
    const int s = j % mix::S;
    if (!tc_wait(full0 + 8 * s, (uint32_t)((j / mix::S) & 1), p.wait_limit)) return false;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t a0 = sbase + s * C::A_ST, b0 = sbase + C::W_OFF, d = taddr + (uint32_t)((j & 1) * C::NCOL);
#pragma unroll
    for (int kk = 0; kk < KC / 16; ++kk) {
      const uint64_t da = tc_sdesc_sw128_mn(a0 + kk * 2048, KC * 128);
      const uint64_t db = tc_sdesc(b0 + kk * 2 * C::LBO_W, C::LBO_W, 128);
      asm volatile(
          "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
          :
          : "r"(d), "l"(da), "l"(db), "r"(C::IDESC), "r"(kk > 0 ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
        mdone0 + 8 * (j & 1)));
    return true;
  };
  int ok = 1, issued = 0, mmas = 0;
  if (tid == 0) {
    for (; issued < min(mix::S, n_my); ++issued) issue(issued);
    if (mma(0)) mmas = 1; else ok = 0;
  }
  ok = __syncthreads_and(ok);
  for (int j = 0; j < n_my && ok; ++j) {
    const int t = (int)blockIdx.x + j * (int)gridDim.x;
    const int b = t / tiles_n, n0 = (t - b * tiles_n) * mix::TP;
    const int n = n0 + warp * 32 + lane;
    const bool live = n < p.N;
    // the f32 term of this tile: independent of the MMAs, so its loads go first
    float add[MC];
#pragma unroll
    for (int e = 0; e < MC; ++e) add[e] = 0.f;
    if (p.cadd && live) {
      const float* q = p.cadd + (long long)b * p.sadd + n;
#pragma unroll
      for (int e = 0; e < MC; ++e) add[e] = __ldg(q + (long long)e * p.ldadd);
    } else if (p.cadd_h && live) {
      const bf16* q = p.cadd_h + (long long)b * p.sadd + n;
#pragma unroll
      for (int e = 0; e < MC; ++e) add[e] = __bfloat162float(q[(long long)e * p.ldadd]);
    }
    if (tid == 0 && j + 1 < n_my) {  // next tile into the other accumulator (read out by iteration j - 1)
      if (mma(j + 1)) mmas = j + 2; else ok = 0;
    }
    if (!tc_wait(mdone0 + 8 * (j & 1), (uint32_t)((j >> 1) & 1), p.wait_limit)) ok = 0;
    if (!__syncthreads_and(ok)) {
      ok = 0;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (tid == 0 && issued < n_my) issue(issued++);  // tile j's stage is free again
    const float bn = (p.bias_n && live) ? __ldg(p.bias_n + n) : 0.f;
#pragma unroll
    for (int c0 = 0; c0 < MC; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)((j & 1) * C::NCOL + c0), v);
      if (!live) continue;
      // output rows walked by pointer increments (one 64-bit add per element and array)
      bf16* pq = p.pre ? p.pre + (long long)b * p.spre + (long long)c0 * p.ldpre + n : nullptr;
      const long long o0 = (long long)b * p.sc + (long long)c0 * p.ldc + n;
      float* fq = p.outf ? p.outf + o0 : nullptr;
      bf16* hq = p.outh ? p.outh + o0 : nullptr;
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int m = c0 + e;
        float y = p.alpha * __uint_as_float(v[e]) + add[m] + s_bias[m] + bn;
        if (pq) {
          *pq = __float2bfloat16_rn(y);
          pq += p.ldpre;
        }
        if (p.act == 1) y = fq ? gelu_f(y) : gelu_bf16out(y);
        if (fq) {
          *fq = y;
          fq += p.ldc;
        }
        if (hq) {
          *hq = __float2bfloat16_rn(y);
          hq += p.ldc;
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();  // accumulator j & 1 read out before tile j + 2's MMAs overwrite it
  }
  if (tid == 0) {
    if (!ok && mmas > 0)  // let issued MMAs drain before the TMEM goes
      tc_wait(mdone0 + 8 * ((mmas - 1) & 1), (uint32_t)(((mmas - 1) >> 1) & 1), p.wait_limit);
    for (int t = mmas; t < issued; ++t)  // copies still in flight after a failure
      tc_wait(full0 + 8 * (t % mix::S), (uint32_t)((t / mix::S) & 1), p.wait_limit);
    if (!ok) atomicExch(&g_tc_error, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(2 * C::NCOL));
}

// The mixing kernel takes: one weight for the whole batch (sa == 0), X (B operand,
// tb == 0) pixel-contiguous with the designs back to back (sb == K * ldb), K and M in
// {32, 64}, a plain or fused epilogue without atomics or split-K, 16-byte aligned rows.
bool mix_eligible(const GemmP& p) {
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0u; };
  return !p.tb && !p.atomic && p.splitk == 1 && p.sa == 0 && (p.K == 32 || p.K == 64) && (p.M == 32 || p.M == 64) &&
         p.N >= 64 && p.ldb % 8 == 0 && p.sb == (long long)p.K * p.ldb && al(p.B) &&
         (long long)p.batch * p.K <= (1LL << 31) - 1;
}

template <int KC, int MC>
int launch_mix_kc_mc(const GemmP& p, cudaStream_t st) {
  using C = MixCfg<KC, MC>;
  static int per_sm = 0;
  if (per_sm == 0) {
    if (cudaFuncSetAttribute(mix_tc_kernel<KC, MC>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM) !=
            cudaSuccess ||
        cudaFuncSetAttribute(mix_tc_kernel<KC, MC>, cudaFuncAttributePreferredSharedMemoryCarveout, 100) !=
            cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_gemm_bf16: cannot configure the mixing kernel's shared memory");
    // resident CTAs per SM from the kernel's registers (allocated per warp in units of
    // 256), its shared memory (1 KB reserved per CTA) and the 512 TMEM columns
    cudaFuncAttributes fa;
    int dev = 0, smem_sm = 0;
    if (cudaFuncGetAttributes(&fa, mix_tc_kernel<KC, MC>) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_gemm_bf16: cannot query the mixing kernel's resources");
    const int regs_cta = ((fa.numRegs * 32 + 255) / 256 * 256) * (mix::THREADS / 32);
    const int by_regs = 65536 / max(1, regs_cta), by_smem = smem_sm / (C::SMEM + (int)fa.sharedSizeBytes + 1024);
    per_sm = max(1, min(min(by_regs, by_smem), min(8, 512 / (2 * C::NCOL))));
  }
  alignas(64) CUtensorMap mx;
  if (!make_map(&mx, p.B, (long long)p.batch * KC, p.N, p.ldb, KC)) return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles_n = (int)ceil_div(p.N, mix::TP);
  const long long n_tiles = (long long)p.batch * tiles_n;
  if (n_tiles > (1LL << 31) - 1) return 0;
  const int grid = (int)(n_tiles < (long long)sms * per_sm ? n_tiles : (long long)sms * per_sm);
  mix_tc_kernel<KC, MC><<<grid, mix::THREADS, C::SMEM, st>>>(mx, p, (int)n_tiles, tiles_n);
  const int rc = check_launch("bz_gemm_bf16");
  return rc == BZ_OK ? 1 : rc;
}

// 1: launched; 0: not applicable (caller uses another kernel); <0: error status.
int launch_mix(const GemmP& p, cudaStream_t st) {
  if (p.K == 32) return p.M == 32 ? launch_mix_kc_mc<32, 32>(p, st) : launch_mix_kc_mc<32, 64>(p, st);
  return p.M == 32 ? launch_mix_kc_mc<64, 32>(p, st) : launch_mix_kc_mc<64, 64>(p, st);
}

// ---- tcgen05 weight gradients: outf[M][N] += alpha sum_b A[b] (M x K) B[b]^T (K x N) -----
// The surrogate's 1x1-layer weight gradients: both operands are activations with the K
// pixels contiguous (K-major), M (<= 128) and N (16..128) channel rows, summed over the
// pixels and the batch. A persistent CTA takes a contiguous range of (design, 64-pixel)
// items, loads each item's M + N rows by TMA (128-byte swizzle) through a four-stage ring
// and accumulates all of them into one TMEM tile with 128 x N x 16 MMAs (rows M..127 of
// the A stage are never loaded: their accumulator rows are not read); at the end the
// warps holding rows below M add alpha times their rows to outf atomically. Memory-bound:
// (M + N) x 2 bytes per pixel and design.
namespace wg {
constexpr int S = 4, BK = 64, THREADS = 128, A_ST = 128 * BK * 2;
}

template <int NC>
__global__ void __launch_bounds__(wg::THREADS) wgrad_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                                                              const __grid_constant__ CUtensorMap tmB, GemmP p,
                                                              int n_items, int items_b) {
  constexpr int B_ST = NC * wg::BK * 2, STAGE = wg::A_ST + B_ST, NCOL = NC < 32 ? 32 : NC;
  constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NC >> 3) << 17) | (8u << 24);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* bar = smem + wg::S * STAGE;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 8 * (2 * wg::S + 1));
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t full0 = static_cast<uint32_t>(__cvta_generic_to_shared(bar));
  const uint32_t empty0 = full0 + 8 * wg::S, done = full0 + 16 * wg::S;
  const uint32_t tx = (uint32_t)(p.M + NC) * wg::BK * 2;
  // this CTA's items [i0, i1): item i = (design i / items_b, pixels 64 (i % items_b) ...)
  const int per = (n_items + (int)gridDim.x - 1) / (int)gridDim.x;
  const int i0 = min(n_items, (int)blockIdx.x * per), i1 = min(n_items, i0 + per), nt = i1 - i0;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot))),
                 "r"(NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < 2 * wg::S + 1; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(full0 + 8 * i));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t taddr = *tmem_slot;

  int ok = 1;
  if (tid == 0 && nt > 0) {
    auto issue = [&](int t) {  // item i0 + t into stage t % S
      const int i = i0 + t, b = i / items_b, k0 = (i - b * items_b) * wg::BK;
      const uint32_t st = sbase + (t % wg::S) * STAGE, fb = full0 + 8 * (t % wg::S);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(tx) : "memory");
      tma_load_2d(st, &tmA, k0, b * p.M, fb);
      tma_load_2d(st + wg::A_ST, &tmB, k0, b * NC, fb);
    };
    int issued = 0, consumed = 0;
    for (; issued < min(wg::S, nt); ++issued) issue(issued);
    for (int it = 0; it < nt; ++it) {
      const int s = it % wg::S;
      if (!tc_wait(full0 + 8 * s, (uint32_t)((it / wg::S) & 1), p.wait_limit)) {
        ok = 0;
        break;
      }
      consumed = it + 1;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t a0 = sbase + s * STAGE, b0 = a0 + wg::A_ST;
#pragma unroll
      for (int kk = 0; kk < wg::BK / 16; ++kk) {
        const uint64_t da = tc_sdesc_sw128(a0 + kk * 32);
        const uint64_t db = tc_sdesc_sw128(b0 + kk * 32);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            :
            : "r"(taddr), "l"(da), "l"(db), "r"(IDESC), "r"((it > 0 || kk > 0) ? 1u : 0u), "r"(0u), "r"(0u),
              "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          empty0 + 8 * s));
      if (it >= 1 && issued < nt) {  // refill the previous stage once its MMAs are done
        const int sp = (it - 1) % wg::S;
        if (!tc_wait(empty0 + 8 * sp, (uint32_t)(((it - 1) / wg::S) & 1), p.wait_limit)) {
          ok = 0;
          break;
        }
        issue(issued++);
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(done));
    for (int t = consumed; t < issued; ++t)  // copies still in flight after a failure
      tc_wait(full0 + 8 * (t % wg::S), (uint32_t)((t / wg::S) & 1), p.wait_limit);
  }
  ok = __syncthreads_and(ok);
  if (nt > 0 && !tc_wait(done, 0u, p.wait_limit)) ok = 0;
  ok = __syncthreads_and(ok);
  if (!ok && tid == 0) atomicExch(&g_tc_error, 1);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (ok && nt > 0 && warp * 32 < p.M) {  // warps holding accumulator rows below M
    const int m = warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (m < p.M) {
#pragma unroll
        for (int e = 0; e < 32 && c0 + e < NC; ++e) atomicAdd(p.outf + (long long)m * p.ldc + c0 + e, p.alpha * __uint_as_float(v[e]));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(NCOL));
}

// The weight-gradient kernel takes: ta = 0, tb = 1, atomic with sc = 0 (a sum over the
// batch; any split-K request is met by its own split over items), M <= 128, N = 32 or 64,
// K >= 64, rows 16-byte aligned with the designs back to back (sa = M lda, sb = N ldb).
bool wgrad_eligible(const GemmP& p) {
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0u; };
  return !p.ta && p.tb && p.atomic && p.sc == 0 && p.outf && p.M >= 1 && p.M <= 128 && (p.N == 32 || p.N == 64) &&
         p.K >= 64 && p.lda % 8 == 0 && p.ldb % 8 == 0 && p.sa == (long long)p.M * p.lda &&
         p.sb == (long long)p.N * p.ldb && al(p.A) && al(p.B) && (long long)p.batch * 128 <= (1LL << 31) - 1;
}

template <int NC>
int launch_wgrad_nc(const GemmP& p, cudaStream_t st) {
  constexpr int SMEM = wg::S * (wg::A_ST + NC * wg::BK * 2) + 8 * (2 * wg::S + 1) + 16 + 1024;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(wgrad_tc_kernel<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
      return fail(BZ_ERR_CUDA, "bz_gemm_bf16: cannot configure the weight-gradient kernel's shared memory");
    configured = true;
  }
  alignas(64) CUtensorMap ma, mb;
  if (!make_map(&ma, p.A, (long long)p.batch * p.M, p.K, p.lda, p.M) ||
      !make_map(&mb, p.B, (long long)p.batch * NC, p.K, p.ldb, NC))
    return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int items_b = (int)ceil_div(p.K, wg::BK);
  const long long n_items = (long long)p.batch * items_b;
  if (n_items > (1LL << 31) - 1) return 0;
  const int grid = (int)(n_items < 2LL * sms ? n_items : 2LL * sms);  // two CTAs per SM (80-96 KB each)
  wgrad_tc_kernel<NC><<<grid, wg::THREADS, SMEM, st>>>(ma, mb, p, (int)n_items, items_b);
  const int rc = check_launch("bz_gemm_bf16");
  return rc == BZ_OK ? 1 : rc;
}

// 1: launched; 0: not applicable; <0: error status.
int launch_wgrad(const GemmP& p, cudaStream_t st) {
  return p.N == 32 ? launch_wgrad_nc<32>(p, st) : launch_wgrad_nc<64>(p, st);
}

// ---- spectral channel mixing: O[b][o][k] = sum_c U[b][c][k] * W[k][c][o] (complex) ---
// U, O: [B][C][n_modes][2] bf16 (re, im); W: [n_modes][Ci][Co][2] bf16. A block takes KB
// consecutive modes, so every global access moves KB complex values (16 bytes) per
// channel row instead of one, and stages the modes' weights and a chunk of designs'
// coefficients in shared memory as float2 (mode index fastest, so the lanes of a warp
// read consecutive words). Each thread keeps several outputs in registers; when the
// output index step 256 is a multiple of KB x channels (UNI: channels a power of two up
// to 64), all of a thread's outputs share one weight (forward) or one coefficient row
// (backward) per reduction step, which is then read once. Sums run in the same order
// with the same fused multiply-adds for every block shape.
constexpr int KB = 4;      // consecutive modes per block
constexpr int DB = 16;     // designs per block (forward)
constexpr int DBB = 8;     // designs per shared-memory chunk (backward)
constexpr int SMAXC = 32;  // channels supported by the staged kernels

__device__ __forceinline__ float2 ld_c(const bf16* p) {
  return make_float2(__bfloat162float(p[0]), __bfloat162float(p[1]));
}

__device__ __forceinline__ void st_c(bf16* p, float re, float im) {
  *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(re, im);
}

// grid (ceil(n_modes / KB), ceil(B / DB)), 256 threads
template <bool UNI>
__global__ void __launch_bounds__(256) spectral_fwd_kernel(const bf16* __restrict__ U, const bf16* __restrict__ W,
                                                           bf16* __restrict__ O, int B, int Ci, int Co, int nk) {
  __shared__ float2 sw[SMAXC * SMAXC * KB];  // [c][o][kk]
  __shared__ float2 su[DB * SMAXC * KB];     // [b][c][kk]
  constexpr int NJ = DB * SMAXC * KB / 256;  // outputs per thread
  const int k0 = blockIdx.x * KB, b0 = blockIdx.y * DB;
  const int nkb = min(KB, nk - k0), nb = min(DB, B - b0), CC = Ci * Co;
  for (int t = threadIdx.x; t < KB * CC; t += 256) {  // along o: contiguous reads
    const int kk = t / CC, r = t - kk * CC;
    sw[r * KB + kk] = kk < nkb ? ld_c(W + ((long long)(k0 + kk) * CC + r) * 2) : make_float2(0.f, 0.f);
  }
  for (int t = threadIdx.x; t < nb * Ci * KB; t += 256) {  // KB consecutive modes per channel row
    const int kk = t % KB, bc = t / KB;
    su[t] = kk < nkb ? ld_c(U + (((long long)b0 * Ci + bc) * nk + k0 + kk) * 2) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int n_out = nb * Co * KB;
  int ub[NJ], wo[NJ];
  float re[NJ], im[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {  // output i = (b, o, kk), kk fastest
    const int i = threadIdx.x + 256 * j;
    const int kk = i % KB, bo = i / KB, b = bo / Co, o = bo - b * Co;
    const bool in = i < n_out;
    ub[j] = in ? b * Ci * KB + kk : 0;
    wo[j] = in ? o * KB + kk : 0;
    re[j] = 0.f;
    im[j] = 0.f;
  }
  for (int c = 0; c < Ci; ++c) {
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const float2 w = sw[c * Co * KB + (UNI ? wo[0] : wo[j])];
      const float2 u = su[ub[j] + c * KB];
      re[j] = fmaf(u.x, w.x, fmaf(-u.y, w.y, re[j]));
      im[j] = fmaf(u.x, w.y, fmaf(u.y, w.x, im[j]));
    }
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int i = threadIdx.x + 256 * j;
    const int kk = i % KB, bo = i / KB;
    if (i < n_out && kk < nkb) {
      const int b = bo / Co, o = bo - b * Co;
      st_c(O + (((long long)(b0 + b) * Co + o) * nk + k0 + kk) * 2, re[j], im[j]);
    }
  }
}

// Backward of KB modes: dU[b][c] = sum_o dO[b][o] conj(W[c][o]); dW[c][o] += sum_b dO[b][o]
// conj(U[b][c]) (f32; one block owns its modes' dW, so no atomics). grid ceil(n_modes / KB).
template <bool UNI>
__global__ void __launch_bounds__(256) spectral_bwd_kernel(const bf16* __restrict__ dO, const bf16* __restrict__ U,
                                                           const bf16* __restrict__ W, bf16* __restrict__ dU,
                                                           float* __restrict__ dW, int B, int Ci, int Co, int nk) {
  __shared__ float2 sw[SMAXC * SMAXC * KB];  // [o][c][kk]
  __shared__ float2 su[DBB * SMAXC * KB];    // [b][c][kk]
  __shared__ float2 sg[DBB * SMAXC * KB];    // [b][o][kk]
  constexpr int NW = SMAXC * SMAXC * KB / 256;  // dW outputs per thread
  constexpr int NU = DBB * SMAXC * KB / 256;    // dU outputs per thread and chunk
  const int k0 = blockIdx.x * KB, nkb = min(KB, nk - k0), CC = Ci * Co;
  for (int t = threadIdx.x; t < KB * CC; t += 256) {
    const int kk = t / CC, r = t - kk * CC, c = r / Co, o = r - c * Co;
    sw[(o * Ci + c) * KB + kk] = kk < nkb ? ld_c(W + ((long long)(k0 + kk) * CC + r) * 2) : make_float2(0.f, 0.f);
  }
  // dW outputs i = (c, o, kk), kk fastest
  const int n_w = CC * KB;
  float ar[NW], ai[NW];
#pragma unroll
  for (int j = 0; j < NW; ++j) {
    ar[j] = 0.f;
    ai[j] = 0.f;
  }
  for (int bb = 0; bb < B; bb += DBB) {
    const int nb = min(DBB, B - bb);
    __syncthreads();
    for (int t = threadIdx.x; t < nb * Ci * KB; t += 256) {
      const int kk = t % KB, bc = t / KB;
      su[t] = kk < nkb ? ld_c(U + (((long long)bb * Ci + bc) * nk + k0 + kk) * 2) : make_float2(0.f, 0.f);
    }
    for (int t = threadIdx.x; t < nb * Co * KB; t += 256) {
      const int kk = t % KB, bo = t / KB;
      sg[t] = kk < nkb ? ld_c(dO + (((long long)bb * Co + bo) * nk + k0 + kk) * 2) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // dU outputs i = (b, c, kk), kk fastest
    const int n_u = nb * Ci * KB;
    int gb[NU], wc[NU];
    float ur[NU], ui[NU];
#pragma unroll
    for (int j = 0; j < NU; ++j) {
      const int i = threadIdx.x + 256 * j;
      const int kk = i % KB, bc = i / KB, b = bc / Ci, c = bc - b * Ci;
      const bool in = i < n_u;
      gb[j] = in ? b * Co * KB + kk : 0;
      wc[j] = in ? c * KB + kk : 0;
      ur[j] = 0.f;
      ui[j] = 0.f;
    }
    for (int o = 0; o < Co; ++o) {
#pragma unroll
      for (int j = 0; j < NU; ++j) {
        const float2 w = sw[o * Ci * KB + (UNI ? wc[0] : wc[j])];
        const float2 g = sg[gb[j] + o * KB];
        ur[j] = fmaf(g.x, w.x, fmaf(g.y, w.y, ur[j]));
        ui[j] = fmaf(g.y, w.x, fmaf(-g.x, w.y, ui[j]));
      }
    }
#pragma unroll
    for (int j = 0; j < NU; ++j) {
      const int i = threadIdx.x + 256 * j;
      const int kk = i % KB, bc = i / KB;
      if (i < n_u && kk < nkb) st_c(dU + (((long long)bb * Ci + bc) * nk + k0 + kk) * 2, ur[j], ui[j]);
    }
    // dW: conj(U) dO summed over this chunk's designs, in design order
    for (int b = 0; b < nb; ++b) {
#pragma unroll
      for (int j = 0; j < NW; ++j) {
        const int i = threadIdx.x + 256 * j;
        const int kk = i % KB, co = i / KB, c = co / Co, o = co - c * Co;
        const bool in = i < n_w;
        const float2 g = sg[b * Co * KB + (in ? o * KB + kk : 0)];
        const float2 u = su[b * Ci * KB + (in ? c * KB + kk : 0)];
        ar[j] = fmaf(g.x, u.x, fmaf(g.y, u.y, ar[j]));
        ai[j] = fmaf(g.y, u.x, fmaf(-g.x, u.y, ai[j]));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NW; ++j) {
    const int i = threadIdx.x + 256 * j;
    const int kk = i % KB, co = i / KB;
    if (i < n_w && kk < nkb) {
      const int c = co / Co, o = co - c * Co;
      float* d = dW + ((long long)(k0 + kk) * CC + c * Co + o) * 2;
      d[0] += ar[j];
      d[1] += ai[j];
    }
  }
}

// dx = dy * GELU'(pre); VEC: 8 values per thread and step with 16-byte accesses (all three
// arrays 16-byte aligned, n a multiple of 8).
template <bool VEC>
__global__ void gelu_bwd_kernel(const bf16* __restrict__ dy, const bf16* __restrict__ pre, bf16* __restrict__ dx,
                                long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (VEC) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n / 8; i += stride) {
      const uint4 a = __ldg(reinterpret_cast<const uint4*>(dy) + i), q = __ldg(reinterpret_cast<const uint4*>(pre) + i);
      const __nv_bfloat162* a2 = reinterpret_cast<const __nv_bfloat162*>(&a);
      const __nv_bfloat162* q2 = reinterpret_cast<const __nv_bfloat162*>(&q);
      uint4 r;
      __nv_bfloat162* r2 = reinterpret_cast<__nv_bfloat162*>(&r);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 av = __bfloat1622float2(a2[e]), qv = __bfloat1622float2(q2[e]);
        r2[e] = __floats2bfloat162_rn(av.x * gelu_grad(qv.x), av.y * gelu_grad(qv.y));
      }
      reinterpret_cast<uint4*>(dx)[i] = r;
    }
    return;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    dx[i] = __float2bfloat16_rn(__bfloat162float(dy[i]) * gelu_grad(__bfloat162float(pre[i])));
}

// out[r] = scale * sum_p x[r][p] over rows r of length P (bf16 in, f32 out): one warp per row.
__global__ void row_mean_kernel(const bf16* __restrict__ x, float* __restrict__ out, long long rows, int P,
                                float scale) {
  const long long r = blockIdx.x * (long long)(blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= rows) return;
  const int lane = threadIdx.x & 31;
  float s = 0.f;
  for (int p = lane; p < P; p += 32) s += __bfloat162float(x[r * P + p]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[r] = s * scale;
}

// Sum over rows: out[c] += sum_b sum_p x[b][c][p] (bf16 in, f32 out); one block per
// (c, b) row of P values, reduced in the block and added atomically. VEC: rows 16-byte
// aligned (P a multiple of 8), read 8 values per thread and step.
template <bool VEC>
__global__ void chan_sum_kernel(const bf16* __restrict__ x, float* __restrict__ out, int B, int C, int P) {
  const int c = blockIdx.x, b = blockIdx.y;
  const bf16* row = x + ((long long)b * C + c) * P;
  float s = 0.f;
  if (VEC) {
    for (int p = threadIdx.x; p < P / 8; p += blockDim.x) {
      const uint4 a = __ldg(reinterpret_cast<const uint4*>(row) + p);
      const __nv_bfloat162* a2 = reinterpret_cast<const __nv_bfloat162*>(&a);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 v = __bfloat1622float2(a2[e]);
        s += v.x + v.y;
      }
    }
  } else {
    for (int p = threadIdx.x; p < P; p += blockDim.x) s += __bfloat162float(row[p]);
  }
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(out + c, s);
  }
}

// x[r][p] = g[r] * scale (broadcast of a per-row gradient), bf16 out; VEC: P a multiple of
// 8 and x 16-byte aligned, 8 values per thread and step.
template <bool VEC>
__global__ void row_broadcast_kernel(const float* __restrict__ g, bf16* __restrict__ x, long long rows, int P,
                                     float scale) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (VEC) {
    const int P8 = P / 8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows * P8; i += stride) {
      const __nv_bfloat162 v = __float2bfloat162_rn(__ldg(g + i / P8) * scale);
      uint4 r;
      __nv_bfloat162* r2 = reinterpret_cast<__nv_bfloat162*>(&r);
#pragma unroll
      for (int e = 0; e < 4; ++e) r2[e] = v;
      reinterpret_cast<uint4*>(x)[i] = r;
    }
    return;
  }
  const long long n = rows * P;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    x[i] = __float2bfloat16_rn(g[i / P] * scale);
}

// Adam on f32 master weights; refreshes the bf16 copy used by the kernels.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, bf16* __restrict__ wh, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wn = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wn;
    if (wh) wh[i] = __float2bfloat16_rn(wn);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, bf16* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

unsigned grid_for(long long n, int threads) {
  const long long b = (n + threads - 1) / threads;
  return (unsigned)(b < 148LL * 32 ? (b < 1 ? 1 : b) : 148LL * 32);
}

}  // namespace
}  // namespace bz

extern "C" int bz_gemm_bf16(const bz_gemm* g, void* stream) {
  BZ_REQUIRE(g != nullptr, "bz_gemm_bf16: NULL arguments");
  BZ_REQUIRE(g->M >= 0 && g->N >= 0 && g->K >= 0 && g->batch >= 1 && g->splitk >= 1,
             "bz_gemm_bf16: bad sizes M=%d N=%d K=%d batch=%d splitk=%d", g->M, g->N, g->K, g->batch, g->splitk);
  BZ_REQUIRE(g->A && g->B, "bz_gemm_bf16: NULL operand");
  BZ_REQUIRE(g->outf || g->outh, "bz_gemm_bf16: no output");
  BZ_REQUIRE(!(g->cadd && g->cadd_h), "bz_gemm_bf16: give the added term as f32 or as bf16, not both");
  BZ_REQUIRE(!(g->atomic || g->splitk > 1) || (g->outf && !g->outh && !g->cadd && !g->cadd_h && !g->bias_m && !g->bias_n &&
                                                !g->pre && g->act == 0),
             "bz_gemm_bf16: atomic/split-K output takes a plain f32 product only");
  BZ_REQUIRE(g->splitk == 1 || g->atomic, "bz_gemm_bf16: split-K needs atomic accumulation");
  BZ_REQUIRE(g->act == 0 || g->act == 1, "bz_gemm_bf16: unknown activation %d", g->act);
  BZ_REQUIRE((long long)g->batch * g->splitk <= 65535, "bz_gemm_bf16: batch x splitk above 65535");
  if (g->M == 0 || g->N == 0) return BZ_OK;
  bz::GemmP p;
  p.M = g->M; p.N = g->N; p.K = g->K; p.batch = g->batch; p.splitk = g->splitk; p.act = g->act;
  p.ta = g->ta; p.tb = g->tb; p.atomic = g->atomic;
  p.A = (const bz::bf16*)g->A; p.lda = g->lda; p.sa = g->sa;
  p.B = (const bz::bf16*)g->B; p.ldb = g->ldb; p.sb = g->sb;
  p.alpha = g->alpha;
  p.cadd = g->cadd; p.ldadd = g->ldadd; p.sadd = g->sadd;
  p.cadd_h = (const bz::bf16*)g->cadd_h;
  p.bias_m = g->bias_m; p.bias_n = g->bias_n;
  p.outf = g->outf; p.outh = (bz::bf16*)g->outh; p.ldc = g->ldc; p.sc = g->sc;
  p.pre = (bz::bf16*)g->pre; p.ldpre = g->ldpre; p.spre = g->spre;
  p.wait_limit = bz::tc::WAIT_LIMIT;
  p.withhold = 0;
  cudaStream_t st = bz::as_stream(stream);
  if (g->engine == 0 && bz::tc_eligible(p)) {
    const int t = bz::launch_gemm_tma(p, st);
    if (t != 0) return t > 0 ? BZ_OK : t;
    return bz::launch_gemm_tc(p, st);
  }
  if (g->engine == 0 && bz::wgrad_eligible(p)) {
    const int t = bz::launch_wgrad(p, st);
    if (t != 0) return t > 0 ? BZ_OK : t;
  }
  if (g->engine == 0 && bz::mix_eligible(p)) {
    const int t = bz::launch_mix(p, st);
    if (t != 0) return t > 0 ? BZ_OK : t;
  }
  if (g->engine == 2 && bz::tc_eligible(p)) return bz::launch_gemm_tc(p, st);
  if (g->N <= 32) return bz::launch_gemm<128, 32, 4, 1>(p, st);
  if (g->M <= 32) return bz::launch_gemm<32, 128, 1, 4>(p, st);
  return bz::launch_gemm<128, 128, 2, 4>(p, st);
}

extern "C" int bz_gemm_wait_selftest(const void* A, const void* B, float* C, int32_t wait_limit, void* stream) {
  BZ_REQUIRE(A && B && C, "bz_gemm_wait_selftest: NULL buffer");
  BZ_REQUIRE(wait_limit >= 1, "bz_gemm_wait_selftest: wait_limit must be positive");
  bz::GemmP p = {};
  p.M = 128; p.N = 256; p.K = 64; p.batch = 1; p.splitk = 1;
  p.A = (const bz::bf16*)A; p.lda = 64;
  p.B = (const bz::bf16*)B; p.ldb = 64;
  p.alpha = 1.0f;
  p.outf = C; p.ldc = 256;
  p.wait_limit = wait_limit;
  p.withhold = 1;
  cudaStream_t st = bz::as_stream(stream);
  const int zero = 0;
  if (cudaMemcpyToSymbolAsync(bz::g_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return bz::fail(BZ_ERR_CUDA, "bz_gemm_wait_selftest: cannot reset the error word");
  const int rc = bz::launch_gemm_tc(p, st);
  if (rc != BZ_OK) return rc;
  if (cudaStreamSynchronize(st) != cudaSuccess) return bz::fail(BZ_ERR_CUDA, "bz_gemm_wait_selftest: launch failed");
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, bz::g_tc_error, sizeof(int)) != cudaSuccess)
    return bz::fail(BZ_ERR_CUDA, "bz_gemm_wait_selftest: cannot read the error word");
  if (cudaMemcpyToSymbol(bz::g_tc_error, &zero, sizeof(int)) != cudaSuccess)
    return bz::fail(BZ_ERR_CUDA, "bz_gemm_wait_selftest: cannot reset the error word");
  if (v) return bz::fail(BZ_ERR_TIMEOUT, "bz_gemm_wait_selftest: the withheld slice's wait ran out after %d polls",
                         wait_limit);
  return BZ_OK;
}

extern "C" int bz_gemm_error(int32_t* value, int32_t reset) {
  BZ_REQUIRE(value != nullptr, "bz_gemm_error: NULL value");
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, bz::g_tc_error, sizeof(int)) != cudaSuccess)
    return bz::fail(BZ_ERR_CUDA, "bz_gemm_error: cannot read the error word");
  *value = v;
  if (reset && v) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(bz::g_tc_error, &zero, sizeof(int)) != cudaSuccess)
      return bz::fail(BZ_ERR_CUDA, "bz_gemm_error: cannot reset the error word");
  }
  return BZ_OK;
}

extern "C" int bz_spectral_mix(const void* U, const void* W, void* O, int32_t B, int32_t ci, int32_t co,
                               int32_t n_modes, void* stream) {
  BZ_REQUIRE(U && W && O, "bz_spectral_mix: NULL buffer");
  BZ_REQUIRE(B >= 1 && ci >= 1 && co >= 1 && ci <= bz::SMAXC && co <= bz::SMAXC && n_modes >= 1,
             "bz_spectral_mix: bad sizes (channels up to %d)", bz::SMAXC);
  BZ_REQUIRE(B <= 65535 * bz::DB, "bz_spectral_mix: batch above %d", 65535 * bz::DB);
  const dim3 grid((unsigned)bz::ceil_div(n_modes, bz::KB), (unsigned)bz::ceil_div(B, bz::DB));
  if (256 % (bz::KB * co) == 0)
    bz::spectral_fwd_kernel<true><<<grid, 256, 0, bz::as_stream(stream)>>>((const bz::bf16*)U, (const bz::bf16*)W,
                                                                          (bz::bf16*)O, B, ci, co, n_modes);
  else
    bz::spectral_fwd_kernel<false><<<grid, 256, 0, bz::as_stream(stream)>>>((const bz::bf16*)U, (const bz::bf16*)W,
                                                                           (bz::bf16*)O, B, ci, co, n_modes);
  return bz::check_launch("bz_spectral_mix");
}

extern "C" int bz_spectral_mix_bwd(const void* dO, const void* U, const void* W, void* dU, float* dW, int32_t B,
                                   int32_t ci, int32_t co, int32_t n_modes, void* stream) {
  BZ_REQUIRE(dO && U && W && dU && dW, "bz_spectral_mix_bwd: NULL buffer");
  BZ_REQUIRE(B >= 1 && ci >= 1 && co >= 1 && ci <= bz::SMAXC && co <= bz::SMAXC && n_modes >= 1,
             "bz_spectral_mix_bwd: bad sizes (channels up to %d)", bz::SMAXC);
  const unsigned grid = (unsigned)bz::ceil_div(n_modes, bz::KB);
  if (256 % (bz::KB * ci) == 0)
    bz::spectral_bwd_kernel<true><<<grid, 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)dO, (const bz::bf16*)U, (const bz::bf16*)W, (bz::bf16*)dU, dW, B, ci, co, n_modes);
  else
    bz::spectral_bwd_kernel<false><<<grid, 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)dO, (const bz::bf16*)U, (const bz::bf16*)W, (bz::bf16*)dU, dW, B, ci, co, n_modes);
  return bz::check_launch("bz_spectral_mix_bwd");
}

extern "C" int bz_gelu_bwd(const void* dy, const void* pre, void* dx, int64_t n, void* stream) {
  BZ_REQUIRE(dy && pre && dx && n >= 0, "bz_gelu_bwd: bad arguments");
  if (n == 0) return BZ_OK;
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0u; };
  if (n % 8 == 0 && al(dy) && al(pre) && al(dx))
    bz::gelu_bwd_kernel<true><<<bz::grid_for(n / 8, 256), 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)dy, (const bz::bf16*)pre, (bz::bf16*)dx, n);
  else
    bz::gelu_bwd_kernel<false><<<bz::grid_for(n, 256), 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)dy, (const bz::bf16*)pre, (bz::bf16*)dx, n);
  return bz::check_launch("bz_gelu_bwd");
}

extern "C" int bz_row_mean(const void* x, float* out, int64_t rows, int32_t P, float scale, void* stream) {
  BZ_REQUIRE(x && out && rows >= 0 && P >= 1, "bz_row_mean: bad arguments");
  if (rows == 0) return BZ_OK;
  bz::row_mean_kernel<<<(unsigned)bz::ceil_div(rows, 8), 256, 0, bz::as_stream(stream)>>>((const bz::bf16*)x, out,
                                                                                        rows, P, scale);
  return bz::check_launch("bz_row_mean");
}

extern "C" int bz_row_broadcast(const float* g, void* x, int64_t rows, int32_t P, float scale, void* stream) {
  BZ_REQUIRE(g && x && rows >= 0 && P >= 1, "bz_row_broadcast: bad arguments");
  if (rows == 0) return BZ_OK;
  if (P % 8 == 0 && (reinterpret_cast<uintptr_t>(x) & 15u) == 0u)
    bz::row_broadcast_kernel<true><<<bz::grid_for(rows * (P / 8), 256), 256, 0, bz::as_stream(stream)>>>(
        g, (bz::bf16*)x, rows, P, scale);
  else
    bz::row_broadcast_kernel<false><<<bz::grid_for(rows * P, 256), 256, 0, bz::as_stream(stream)>>>(
        g, (bz::bf16*)x, rows, P, scale);
  return bz::check_launch("bz_row_broadcast");
}

extern "C" int bz_chan_sum(const void* x, float* out, int32_t B, int32_t C, int32_t P, void* stream) {
  BZ_REQUIRE(x && out && B >= 1 && C >= 1 && P >= 1, "bz_chan_sum: bad arguments");
  BZ_REQUIRE(B <= 65535, "bz_chan_sum: B above 65535");
  if (P % 8 == 0 && (reinterpret_cast<uintptr_t>(x) & 15u) == 0u)
    bz::chan_sum_kernel<true><<<dim3((unsigned)C, (unsigned)B), 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)x, out, B, C, P);
  else
    bz::chan_sum_kernel<false><<<dim3((unsigned)C, (unsigned)B), 256, 0, bz::as_stream(stream)>>>(
        (const bz::bf16*)x, out, B, C, P);
  return bz::check_launch("bz_chan_sum");
}

extern "C" int bz_adam(float* w, const float* g, float* m, float* v, void* wh, int64_t n, float lr, float b1,
                       float b2, float eps, int32_t step, float weight_decay, void* stream) {
  BZ_REQUIRE(w && g && m && v && n >= 0 && step >= 1, "bz_adam: bad arguments");
  if (n == 0) return BZ_OK;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  bz::adam_kernel<<<bz::grid_for(n, 256), 256, 0, bz::as_stream(stream)>>>(w, g, m, v, (bz::bf16*)wh, n, lr, b1, b2,
                                                                          eps, c1, c2, weight_decay);
  return bz::check_launch("bz_adam");
}

extern "C" int bz_to_bf16(const float* x, void* y, int64_t n, void* stream) {
  BZ_REQUIRE(x && y && n >= 0, "bz_to_bf16: bad arguments");
  if (n == 0) return BZ_OK;
  bz::to_bf16_kernel<<<bz::grid_for(n, 256), 256, 0, bz::as_stream(stream)>>>(x, (bz::bf16*)y, n);
  return bz::check_launch("bz_to_bf16");
}
