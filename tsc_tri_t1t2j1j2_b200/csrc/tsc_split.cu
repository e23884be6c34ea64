// Split-precision grouped complex GEMM on the 5th-generation tensor cores.
//
// Same task lists as grouped_zgemm (groups = output rectangles, terms
// C += alpha * op(L) * op(R), AXPY/DIAG element terms), computed as Ozaki-style
// splits: every FP64 operand element x is written as three BF16 slices
// x ~ s0 + s1 + s2 (s0 = bf16(x), s1 = bf16(x - s0), s2 = bf16(x - s0 - s1)),
// the slice products whose weight is at least 2^-18 of the leading one --
// (0,0) (0,1) (1,0) (1,1) (0,2) (2,0) -- run as tcgen05.mma kind::f16 with FP32
// accumulators in tensor memory, and the complex product is assembled from four
// real accumulations (Cr += Ar Br - Ai Bi, Ci += Ar Bi + Ai Br).  Each slice
// product is exact in FP32; the accumulation rounds at 2^-24 of the running sum,
// so the result carries about 1e-6 relative error against the FP64 product.
// Element terms and the write-back (beta, partial tiles) are done in FP64.
//
// CTA = one job: a 128 x 64 output tile of one group over a term range.  256
// threads convert the FP64 operands of one K=16 step into the 12 BF16 planes
// (3 slices x re/im, for A and B) of a shared-memory stage in the canonical
// K-major, no-swizzle UMMA layout; one thread issues the step's 24 MMAs and
// commits them to the stage's mbarrier, which frees the stage for the
// conversion three steps later.  Every mbarrier wait is bounded: on timeout
// the kernel records the fact in a device flag, waits (bounded) for its own
// MMAs, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cstdint>

#include "tsc_kernels.cuh"

namespace tsc {

__device__ int g_split_fault = 0;

namespace {

constexpr int SP_TM = 128, SP_TN = 64, SP_TK = 16, SP_STAGES = 3, SP_THREADS = 256;
constexpr int A_PLANE = SP_TM * SP_TK * 2;                     // bytes of one BF16 plane of A
constexpr int B_PLANE = SP_TN * SP_TK * 2;                     // ... of B
constexpr int STAGE_BYTES = 6 * A_PLANE + 6 * B_PLANE;         // 36,864
constexpr int SMEM_BYTES = SP_STAGES * STAGE_BYTES + 128;      // + mbarriers, TMEM slot
constexpr uint32_t TMEM_COLS = 2 * SP_TN;                      // Cr | Ci, FP32
constexpr long long WAIT_LIMIT = 1ll << 20;

// instruction descriptor, kind::f16: D f32, A/B bf16, both K-major, N>>3, M>>4
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SP_TN >> 3) << 17) |
                           ((uint32_t)(SP_TM >> 4) << 24);
constexpr uint32_t IDESC_NEG_A = IDESC | (1u << 13);

// (slice of A, slice of B) products kept
__constant__ int c_pairs[6][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}, {0, 2}, {2, 0}};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of
// 8 rows x 16 bytes stored contiguously (128 B); the two core matrices of one
// K=16 step 128 B apart (leading byte offset), 8-row groups 256 B apart
// (stride byte offset); version 1 (bits 46-47) as sm_100 requires.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// three BF16 slices of x (through FP32, whose 24 bits the slices cover)
__device__ __forceinline__ void split3(double x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  const float f = (float)x;
  a = __float2bfloat16_rn(f);
  const float r1 = f - __bfloat162float(a);
  b = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(b);
  c = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Converts 8 consecutive-k complex values of one row (of A) or column (of B)
// into the six planes (slice-major, re then im) at byte offset `off` of each.
__device__ __forceinline__ void store_chunk(unsigned char* planes, int plane_bytes, int off, const double2* v) {
  uint32_t w[6][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    __nv_bfloat16 a0, b0, c0, a1, b1, c1;
    split3(v[2 * e].x, a0, b0, c0);
    split3(v[2 * e + 1].x, a1, b1, c1);
    w[0][e] = pack2(a0, a1);
    w[2][e] = pack2(b0, b1);
    w[4][e] = pack2(c0, c1);
    split3(v[2 * e].y, a0, b0, c0);
    split3(v[2 * e + 1].y, a1, b1, c1);
    w[1][e] = pack2(a0, a1);
    w[3][e] = pack2(b0, b1);
    w[5][e] = pack2(c0, c1);
  }
#pragma unroll
  for (int p = 0; p < 6; ++p)
    *reinterpret_cast<uint4*>(planes + p * plane_bytes + off) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// byte offset of the chunk (row r, k-chunk kc) inside a plane
__device__ __forceinline__ int chunk_off(int r, int kc) { return (r >> 3) * 256 + kc * 128 + (r & 7) * 16; }

__global__ void __launch_bounds__(SP_THREADS, 2)
grouped_zgemm_split_kernel(const GJob* __restrict__ jobs, const GGroup* __restrict__ groups,
                           const GTerm* __restrict__ terms, Bases bases) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + SP_STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + SP_STAGES * STAGE_BYTES + 64);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const GJob job = jobs[blockIdx.x];
  const GGroup g = groups[job.group];
  const int m0 = job.tm * SP_TM, n0 = job.tn * SP_TN;

  if (tid == 0) {
    for (int s = 0; s < SP_STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  // ---- main loop over the GEMM terms, one K=16 step per pipeline stage -----
  int q = 0;   // steps issued
  bool fault = false;
  for (int ti = job.t0; ti < job.t1 && !fault; ++ti) {
    const GTerm t = terms[ti];
    if (t.kind != TK_GEMM) continue;
    const double2* L = bases.p[t.l_base] + t.l_off;
    const double2* R = bases.p[t.r_base] + t.r_off;
    const int nk = (t.K + SP_TK - 1) / SP_TK;
    for (int kk = 0; kk < nk; ++kk, ++q) {
      const int s = q % SP_STAGES;
      unsigned char* st = smem + s * STAGE_BYTES;
      // the MMAs of step q - STAGES must have finished reading this stage
      const bool ok = q < SP_STAGES || mbar_wait(smem_u32(&bars[s]), (uint32_t)((q / SP_STAGES - 1) & 1));
      // A: op(L), 128 rows x 16 k -> 256 chunks of 8 k, one per thread
      {
        const int r = tid & 127, kc = tid >> 7;
        const int gi = m0 + r, kb = kk * SP_TK + kc * 8;
        double2 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = kb + e;
          double2 x = make_double2(0.0, 0.0);
          if (gi < g.M && k < t.K) {
            x = (t.l_op == OP_N) ? L[(long long)gi + (long long)k * t.l_ld] : L[(long long)k + (long long)gi * t.l_ld];
            if (t.l_op == OP_C) x.y = -x.y;
          }
          v[e] = x;
        }
        store_chunk(st, A_PLANE, chunk_off(r, kc), v);
      }
      // B: alpha * op(R), 16 k x 64 columns -> 128 chunks, threads 0..127
      if (tid < 128) {
        const int c = tid & 63, kc = tid >> 6;
        const int gj = n0 + c, kb = kk * SP_TK + kc * 8;
        double2 v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = kb + e;
          double2 x = make_double2(0.0, 0.0);
          if (gj < g.N && k < t.K) {
            x = (t.r_op == OP_N) ? R[(long long)k + (long long)gj * t.r_ld] : R[(long long)gj + (long long)k * t.r_ld];
            if (t.r_op == OP_C) x.y = -x.y;
          }
          v[e] = make_double2(t.ar * x.x - t.ai * x.y, t.ar * x.y + t.ai * x.x);
        }
        store_chunk(st + 6 * A_PLANE, B_PLANE, chunk_off(c, kc), v);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (__syncthreads_or(!ok)) {   // block-uniform decision
        fault = true;
        break;
      }
      if (tid == 0) {
        fence_after_sync();
        const uint32_t a0 = smem_u32(st), b0 = smem_u32(st + 6 * A_PLANE);
#pragma unroll
        for (int pi = 0; pi < 6; ++pi) {
          const int sa = c_pairs[pi][0], sb = c_pairs[pi][1];
          const uint64_t ar = smem_desc(a0 + (2 * sa) * A_PLANE), ai = smem_desc(a0 + (2 * sa + 1) * A_PLANE);
          const uint64_t br = smem_desc(b0 + (2 * sb) * B_PLANE), bi = smem_desc(b0 + (2 * sb + 1) * B_PLANE);
          const uint32_t first = (q == 0 && pi == 0) ? 0u : 1u;
          umma_bf16(tmem, ar, br, IDESC, first);                  // Cr  = Ar Br
          umma_bf16(tmem, ai, bi, IDESC_NEG_A, 1u);               // Cr -= Ai Bi
          umma_bf16(tmem + SP_TN, ar, bi, IDESC, first);          // Ci  = Ar Bi
          umma_bf16(tmem + SP_TN, ai, br, IDESC, 1u);             // Ci += Ai Br
        }
        umma_commit(smem_u32(&bars[s]));
      }
    }
  }
  // all MMAs of this CTA are complete once the last committed stage arrives
  if (q > 0) {
    const int s = (q - 1) % SP_STAGES;
    if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)(((q - 1) / SP_STAGES) & 1))) fault = true;
  }
  fault = __syncthreads_or(fault);
  fence_after_sync();

  if (!fault) {
    // ---- epilogue: warp w reads TMEM lanes 32*(w%4).., column half w/4 --------
    const int quad = warp & 3, half = warp >> 2;
    const int row = m0 + quad * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16);
    const bool partial = job.part >= 0;
    double2* C = partial ? bases.part + job.part_off : bases.p[g.c_base] + g.c_off;
    const long long ldc = partial ? g.M : g.c_ld;
    const bool acc_old = !partial && g.beta;
#pragma unroll 1
    for (int cb = 0; cb < 2; ++cb) {
      const int c0 = half * 32 + cb * 16;
      float vr[16], vi[16];
      __syncwarp();
      if (q > 0) {
        tmem_ld16(lane_base + c0, vr);
        tmem_ld16(lane_base + SP_TN + c0, vi);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0.f;
      }
      double cr[16], ci[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        cr[j] = vr[j];
        ci[j] = vi[j];
      }
      // element terms (AXPY / DIAG) in FP64, as grouped_zgemm applies them
      for (int ti = job.t0; ti < job.t1; ++ti) {
        const GTerm t = terms[ti];
        if (t.kind == TK_GEMM) continue;
        const double2* R = bases.p[t.r_base] + t.r_off;
        const int rr = row - t.r0;
        if (row >= g.M || rr < 0 || rr >= t.rm) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j, cc = col - t.c0;
          if (col >= g.N || cc < 0 || cc >= t.rn) continue;
          double xr, xi;
          if (t.kind == TK_AXPY) {
            const double2 x = (t.r_op == OP_N) ? R[(long long)rr + (long long)cc * t.r_ld]
                                               : R[(long long)cc + (long long)rr * t.r_ld];
            xr = x.x;
            xi = (t.r_op == OP_C) ? -x.y : x.y;
          } else {
            if (rr != cc) continue;
            xr = 1.0;
            xi = 0.0;
          }
          cr[j] += t.ar * xr - t.ai * xi;
          ci[j] += t.ar * xi + t.ai * xr;
        }
      }
      if (row < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          if (col >= g.N) continue;
          double2* p = C + (long long)row + (long long)col * ldc;
          double2 v = make_double2(cr[j], ci[j]);
          if (acc_old) {
            const double2 o = *p;
            v.x += o.x;
            v.y += o.y;
          }
          *p = v;
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_split_fault, 1);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

cudaError_t launch_grouped_zgemm_split(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms,
                                       Bases bases, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(grouped_zgemm_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SMEM_BYTES);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  grouped_zgemm_split_kernel<<<njobs, SP_THREADS, SMEM_BYTES, st>>>(jobs, groups, terms, bases);
  return cudaGetLastError();
}

cudaError_t split_fault_flag(int* host_flag, int clear) {
  cudaError_t e = cudaMemcpyFromSymbol(host_flag, g_split_fault, sizeof(int));
  if (e != cudaSuccess || !clear) return e;
  const int zero = 0;
  return cudaMemcpyToSymbol(g_split_fault, &zero, sizeof(int));
}

}  // namespace tsc
