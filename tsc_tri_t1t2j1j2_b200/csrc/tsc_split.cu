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
// product is exact in FP32, but every MMA that adds into an FP32 accumulator
// loses a biased part of its last place, so one long chain gathers an error that
// grows like K (5.5e-5 at K=4096 in one accumulator).  Hence two accumulators
// per output -- the (0,0) pair alone ("hi") and the five pairs 2^-8 smaller
// ("lo") -- restarted every SP_SEG K steps; the epilogue adds each segment into
// the output in FP64.  Element terms and the write-back (beta, partial tiles)
// are done in FP64.
//
// Operands arrive pre-sliced.  Every GEMM operand is a view -- an operator
// block (with the term's coefficient folded in, sliced once per superblock; or,
// with term_alpha, shared by all terms of that operator, the epilogue then
// scaling each term's own segments by its coefficient), a
// rectangle of the input vector (sliced once per call by slice_tiles_kernel),
// or a phase-1 intermediate (sliced by the phase-1 launch's own epilogue) --
// stored as stage tiles: six BF16 planes in the canonical K-major, no-swizzle
// UMMA layout, A tiles 128 x 16 (24 KB), B tiles 16 x 64 (12 KB).
//
// Persistent and warp-specialised: one CTA per SM walks the jobs blockIdx.x,
// +gridDim.x, ... (128 x 64 output tiles of a group over a term range, in
// longest-first order).  One producer lane streams the K steps, each an A and a
// B tile brought into a shared-memory stage by two bulk asynchronous copies
// that complete on the stage's full barrier; one lane of the MMA warp issues
// the step's 24 MMAs into one of two TMEM accumulators and commits them to the
// stage's empty barrier (and, after a segment's last step, to the
// accumulator's full barrier); 8 epilogue warps (two per TMEM lane quadrant,
// 32 columns each) drain the other accumulator into the tile in FP64 (the first segment with beta and the element terms,
// later ones adding to it) while the next segment runs.
// Every mbarrier wait is bounded (wait_limit polls, a launch argument): on
// timeout the kernel raises a CTA abort flag and the caller's fault word, waits
// for its own MMAs (a fixed, longer bound: issued MMAs always complete), frees
// its tensor memory and returns.
#include <cuda_bf16.h>
#include <cstdint>

#include "tsc_kernels.cuh"

namespace tsc {

namespace {

constexpr int SP_TM = 128, SP_TN = 64, SP_TK = 16, SP_STAGES = 5;
constexpr int SP_PRODUCER_WARP = 0, SP_MMA_WARP = 1;            // warps 2..9: epilogue
constexpr int SP_EPI_WARPS = 8;   // two per TMEM lane quadrant, each draining 32 of the tile's 64 columns
constexpr int SP_THREADS = (2 + SP_EPI_WARPS) * 32;
constexpr int A_PLANE = SP_TM * SP_TK * 2;                     // bytes of one BF16 plane of A
constexpr int B_PLANE = SP_TN * SP_TK * 2;                     // ... of B
constexpr int STAGE_BYTES = 6 * A_PLANE + 6 * B_PLANE;         // 36,864
constexpr int SMEM_BYTES = SP_STAGES * STAGE_BYTES + 256;      // + mbarriers, TMEM slot, abort flag
static_assert(6 * A_PLANE == 2 * SPLIT_UNIT && 6 * B_PLANE == SPLIT_UNIT, "stage tiles are the arena tiles");
// Two accumulators (double buffer), each [Cr hi | Ci hi | Cr lo | Ci lo]: the
// (0,0) slice pair alone in "hi", the five smaller pairs in "lo".  Both restart
// every SP_SEG K steps; the epilogue adds each segment into the output in FP64,
// so no FP32 chain in tensor memory is longer than 2 * SP_SEG MMAs (hi).
constexpr int SP_SEG = 8;
constexpr uint32_t TMEM_COLS = 8 * SP_TN;                      // 512: the whole of an SM's tensor memory
// polls of the final wait for the CTA's own MMAs before tensor memory is freed
constexpr long long FIN_WAIT_LIMIT = 1ll << 24;

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

// Bounded wait on an mbarrier phase (at most `limit` polls); gives up early
// when another role of the CTA has raised the abort flag.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, long long limit) {
  for (long long i = 0; i < limit; ++i) {
    if (abort_flag && (i & 1023) == 1023 && *abort_flag) return false;
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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// the same load without its wait: several in flight, then one tmem_wait_ld()
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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

// Pre-slices one stage tile of an operand view (the slice kernel below): the
// tile's chunk `chunk` -- 8 consecutive k of one row of op(X) (A role, chunks
// 0..255 of a 128 x 16 tile) or of one column (B role, chunks 0..127 of a
// 16 x 64 tile) -- times the view's coefficient, into the tile's six planes.
__device__ __forceinline__ void slice_chunk(const SView& v, const double2* X, int t, int ks, int chunk,
                                            unsigned char* tile) {
  double2 x[8];
  const bool a_role = v.role == 0;
  const int r = a_role ? (chunk & 127) : (chunk & 63);
  const int kc = a_role ? (chunk >> 7) : (chunk >> 6);
  const int g = t * (a_role ? SP_TM : SP_TN) + r;   // row (A) or column (B) of op(X)
  const int kb = ks * SP_TK + kc * 8;
  const int gmax = a_role ? v.rows : v.cols, kmax = a_role ? v.cols : v.rows;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int k = kb + e;
    double2 y = make_double2(0.0, 0.0);
    if (g < gmax && k < kmax) {
      // A: op(X)[g][k];  B: op(X)[k][g];  op N reads X as stored, op C its conjugate transpose
      const long long i = a_role ? (v.op == OP_N ? (long long)g + (long long)k * v.ld : (long long)k + (long long)g * v.ld)
                                 : (v.op == OP_N ? (long long)k + (long long)g * v.ld : (long long)g + (long long)k * v.ld);
      y = X[i];
      if (v.op == OP_C) y.y = -y.y;
    }
    x[e] = make_double2(v.ar * y.x - v.ai * y.y, v.ar * y.y + v.ai * y.x);
  }
  store_chunk(tile, a_role ? A_PLANE : B_PLANE, chunk_off(r, kc), x);
}

__global__ void __launch_bounds__(256) slice_tiles_kernel(const SView* __restrict__ views,
                                                          const STile* __restrict__ tiles, const double2* in,
                                                          unsigned char* arena, long long arena_units) {
  const STile tl = tiles[blockIdx.x];
  const SView v = views[tl.view];
  const double2* X = v.from_in ? in + v.src : reinterpret_cast<const double2*>((uintptr_t)v.src * sizeof(double2));
  const long long unit = v.dst + (long long)(tl.t * v.nks + tl.ks) * (v.role == 0 ? 2 : 1);
  if (unit < 0 || unit + (v.role == 0 ? 2 : 1) > arena_units) return;   // never outside the arena
  unsigned char* tile = arena + unit * SPLIT_UNIT;
  const int nchunk = v.role == 0 ? 256 : 128;
  if ((int)threadIdx.x < nchunk) slice_chunk(v, X, tl.t, tl.ks, threadIdx.x, tile);
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bulk asynchronous copy global -> shared (no tensor map), completing on an mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// number of K=16 steps of a job (0: only element terms)
__device__ __forceinline__ int job_steps(const GJob& job, const GTerm* terms) {
  int n = 0;
  for (int ti = job.t0; ti < job.t1; ++ti) {
    const GTerm t = terms[ti];
    if (t.kind == TK_GEMM && t.K > 0) n += (t.K + SP_TK - 1) / SP_TK;
  }
  return n;
}

// number of accumulator segments of a job: SP_SEG steps each over the job's
// steps in order, or, with term_alpha, over each GEMM term's steps alone (a
// segment then belongs to one term and the epilogue applies its coefficient)
__device__ __forceinline__ int job_segments(const GJob& job, const GTerm* terms, int term_alpha) {
  if (!term_alpha) return (job_steps(job, terms) + SP_SEG - 1) / SP_SEG;
  int n = 0;
  for (int ti = job.t0; ti < job.t1; ++ti) {
    const GTerm t = terms[ti];
    if (t.kind == TK_GEMM && t.K > 0) n += ((t.K + SP_TK - 1) / SP_TK + SP_SEG - 1) / SP_SEG;
  }
  return n;
}

// Persistent, warp-specialised (roles as described at the top of the file):
// warp 0 streams the stages, warp 1 issues the MMAs into one of two TMEM
// accumulators, warps 2..9 drain the other accumulator into the outputs.
__global__ void __launch_bounds__(SP_THREADS, 1)
grouped_zgemm_split_kernel(const GJob* __restrict__ jobs, int njobs, const GGroup* __restrict__ groups,
                           const GTerm* __restrict__ terms, Bases bases, SplitArenas arenas, int* fault,
                           long long wait_limit, int term_alpha) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + SP_STAGES * STAGE_BYTES);
  uint64_t* empty = full + SP_STAGES;
  uint64_t* accf = empty + SP_STAGES;
  uint64_t* acce = accf + 2;
  uint64_t* fin = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < SP_STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])) : "memory");
    }
    for (int a = 0; a < 2; ++a) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf[a])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acce[a])), "r"(SP_EPI_WARPS) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(fin)) : "memory");
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == SP_MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(fault, 1);
  };

  if (warp == SP_PRODUCER_WARP) {
    // ---------------------------------------------------------------- producer
    // One lane streams the CTA's K steps: per step, the A tile (24 KB) and the
    // B tile (12 KB) of the term's pre-sliced operand views, by two bulk copies
    // that complete on the stage's full barrier.
    if (lane == 0) {
      int last[SP_STAGES];   // last fill issued into each stage (-1: none)
#pragma unroll
      for (int s = 0; s < SP_STAGES; ++s) last[s] = -1;
      int q = 0;
      bool ok = true;
      for (int jb = blockIdx.x; jb < njobs && ok; jb += gridDim.x) {
        const GJob job = jobs[jb];
        for (int ti = job.t0; ti < job.t1 && ok; ++ti) {
          const GTerm t = terms[ti];
          if (t.kind != TK_GEMM || t.K <= 0) continue;
          const int nk = (t.K + SP_TK - 1) / SP_TK;
          // A tile (tm, kk) of the A view at units l_off + (tm * nks + kk) * 2; B tile (tn, kk) at r_off + tn * nks + kk
          const long long ua = t.l_off + 2ll * job.tm * t.l_ld, ub = t.r_off + (long long)job.tn * t.r_ld;
          // every tile this term will copy lies inside its arena, or the CTA stops with a fault
          if (t.l_base > 2 || t.r_base > 2 || ua < 0 || ub < 0 || ua + 2ll * nk > arenas.units[t.l_base] ||
              ub + nk > arenas.units[t.r_base]) {
            ok = false;
            break;
          }
          const unsigned char* A = arenas.a[t.l_base] + ua * SPLIT_UNIT;
          const unsigned char* B = arenas.a[t.r_base] + ub * SPLIT_UNIT;
          for (int kk = 0; kk < nk; ++kk, ++q) {
            const int s = q % SP_STAGES;
            if (q >= SP_STAGES &&
                !mbar_wait(smem_u32(&empty[s]), (uint32_t)((q / SP_STAGES - 1) & 1), abort_flag, wait_limit)) {
              ok = false;
              break;
            }
            const uint32_t st0 = smem_u32(smem + s * STAGE_BYTES), fb = smem_u32(&full[s]);
            mbar_arrive_expect_tx(fb, STAGE_BYTES);
            bulk_g2s(st0, A + 2ll * kk * SPLIT_UNIT, 6 * A_PLANE, fb);
            bulk_g2s(st0 + 6 * A_PLANE, B + (long long)kk * SPLIT_UNIT, 6 * B_PLANE, fb);
            last[s] = q;
          }
        }
      }
      if (!ok) fail();
      // every copy issued here has landed before the CTA leaves, consumed or not
      for (int s = 0; s < SP_STAGES; ++s)
        if (last[s] >= 0 &&
            !mbar_wait(smem_u32(&full[s]), (uint32_t)((last[s] / SP_STAGES) & 1), nullptr, FIN_WAIT_LIMIT))
          fail();
    }
    __syncwarp();
  } else if (warp == SP_MMA_WARP) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      int q = 0, sg = 0;   // stage use, accumulator segment (over the CTA's jobs)
      bool ok = true;
      for (int jb = blockIdx.x; jb < njobs && ok; jb += gridDim.x) {
        const GJob job = jobs[jb];
        const int nst = job_steps(job, terms);
        int i = 0, si = 0;   // step of the job, step within the current segment
        for (int ti = job.t0; ti < job.t1 && ok; ++ti) {
          const GTerm t = terms[ti];
          if (t.kind != TK_GEMM || t.K <= 0) continue;
          const int nk = (t.K + SP_TK - 1) / SP_TK;
          for (int kk = 0; kk < nk; ++kk, ++i, ++q) {
            const int a = sg & 1, ua = sg >> 1;
            if (si == 0) {   // a segment starts: wait until the epilogue has drained this accumulator
              if (ua >= 1 && !mbar_wait(smem_u32(&acce[a]), (uint32_t)((ua - 1) & 1), abort_flag, wait_limit)) {
                ok = false;
                break;
              }
              fence_after_sync();
            }
            const uint32_t dhr = tmem + a * (4 * SP_TN), dhi = dhr + SP_TN, dlr = dhr + 2 * SP_TN, dli = dhr + 3 * SP_TN;
            const int s = q % SP_STAGES;
            if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((q / SP_STAGES) & 1), abort_flag, wait_limit)) {
              ok = false;
              break;
            }
            fence_after_sync();
            const uint32_t a0 = smem_u32(smem + s * STAGE_BYTES), b0 = a0 + 6 * A_PLANE;
#pragma unroll
            for (int pi = 0; pi < 6; ++pi) {
              const int sa = c_pairs[pi][0], sb = c_pairs[pi][1];
              const uint64_t ar = smem_desc(a0 + (2 * sa) * A_PLANE), ai = smem_desc(a0 + (2 * sa + 1) * A_PLANE);
              const uint64_t br = smem_desc(b0 + (2 * sb) * B_PLANE), bi = smem_desc(b0 + (2 * sb + 1) * B_PLANE);
              const uint32_t dcr = pi == 0 ? dhr : dlr, dci = pi == 0 ? dhi : dli;
              const uint32_t first = (si == 0 && pi <= 1) ? 0u : 1u;   // first write of hi (pi 0) and lo (pi 1)
              umma_bf16(dcr, ar, br, IDESC, first);          // Cr  = Ar Br
              umma_bf16(dcr, ai, bi, IDESC_NEG_A, 1u);       // Cr -= Ai Bi
              umma_bf16(dci, ar, bi, IDESC, first);          // Ci  = Ar Bi
              umma_bf16(dci, ai, br, IDESC, 1u);             // Ci += Ai Br
            }
            umma_commit(smem_u32(&empty[s]));
            ++si;
            if (si == SP_SEG || i == nst - 1 || (term_alpha && kk == nk - 1)) {   // segment complete: to the epilogue
              umma_commit(smem_u32(&accf[a]));
              sg++;
              si = 0;
            }
          }
        }
      }
      if (!ok) fail();
      // every MMA issued here has completed before the accumulators are freed
      umma_commit(smem_u32(fin));
      if (!mbar_wait(smem_u32(fin), 0u, nullptr, FIN_WAIT_LIMIT)) fail();
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------------- epilogue
    constexpr int NCB = SP_TN / 16;          // 8-column chunks of one epilogue warp
    const int quad = warp & 3;               // TMEM lane quadrant this warp may read
    const int cb0 = ((warp - 2) >> 2) * NCB; // its half of the tile's 8-column chunks
    int sg = 0;
    bool ok = true;
    for (int jb = blockIdx.x; jb < njobs && ok; jb += gridDim.x) {
      const GJob job = jobs[jb];
      const GGroup g = groups[job.group];
      const int nseg = job_segments(job, terms, term_alpha);
      const int m0 = job.tm * SP_TM, n0 = job.tn * SP_TN;
      const int row = m0 + quad * 32 + lane;
      const bool partial = job.part >= 0;
      double2* C = partial ? bases.part + job.part_off : bases.p[g.c_base] + g.c_off;
      const long long ldc = partial ? g.M : g.c_ld;
      const bool acc_old = !partial && g.beta;
      const bool slice_out = !partial && g.s_off >= 0;
      const int s_nks = (g.N + SP_TK - 1) / SP_TK;
      int ecur = job.t0, erem = 0;         // term_alpha: the segment's term and its steps not yet covered
      double alr = 1.0, ali = 0.0;         // ... and its coefficient
      // the job's segments summed in FP64 registers (this lane's row, the warp's 32 columns);
      // the output tile is then written once
      double accr[NCB][8], acci[NCB][8];
#pragma unroll
      for (int c = 0; c < NCB; ++c)
#pragma unroll
        for (int j = 0; j < 8; ++j) accr[c][j] = acci[c][j] = 0.0;
      for (int sgi = 0; sgi < nseg; ++sgi) {
        const int a = sg & 1, ua = sg >> 1;
        if (term_alpha) {
          while (erem == 0 && ecur < job.t1) {
            const GTerm t = terms[ecur++];
            if (t.kind == TK_GEMM && t.K > 0) {
              erem = (t.K + SP_TK - 1) / SP_TK;
              alr = t.ar;
              ali = t.ai;
            }
          }
          erem -= erem < SP_SEG ? erem : SP_SEG;
        }
        // warp-uniform: the tensor-memory loads below need every lane
        if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&accf[a]), (uint32_t)(ua & 1), abort_flag, wait_limit))) {
          fail();
          ok = false;
          break;
        }
        fence_after_sync();
        const uint32_t lane_base = tmem + a * (4 * SP_TN) + ((uint32_t)(quad * 32) << 16);
#pragma unroll
        for (int c = 0; c < NCB; ++c) {
          const int c0 = (cb0 + c) * 8;
          uint32_t hr[8], hi[8], lr[8], li[8];
          tmem_ld8_nowait(lane_base + c0, hr);
          tmem_ld8_nowait(lane_base + SP_TN + c0, hi);
          tmem_ld8_nowait(lane_base + 2 * SP_TN + c0, lr);
          tmem_ld8_nowait(lane_base + 3 * SP_TN + c0, li);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double sr = (double)__uint_as_float(hr[j]) + (double)__uint_as_float(lr[j]);
            const double si = (double)__uint_as_float(hi[j]) + (double)__uint_as_float(li[j]);
            accr[c][j] += alr * sr - ali * si;
            acci[c][j] += alr * si + ali * sr;
          }
        }
        // this warp's part of the accumulator is read out: hand it back to the MMA warp
        fence_before_sync();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&acce[a]));
        sg++;
      }
      if (!ok) break;
      // element terms (AXPY / DIAG) in FP64, as grouped_zgemm applies them
      for (int ti = job.t0; ti < job.t1; ++ti) {
        const GTerm t = terms[ti];
        if (t.kind == TK_GEMM) continue;
        const double2* R = bases.p[t.r_base] + t.r_off;
        const int rr = row - t.r0;
        if (row >= g.M || rr < 0 || rr >= t.rm) continue;
#pragma unroll
        for (int c = 0; c < NCB; ++c)
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int col = n0 + (cb0 + c) * 8 + j, cc = col - t.c0;
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
            accr[c][j] += t.ar * xr - t.ai * xi;
            acci[c][j] += t.ar * xi + t.ai * xr;
          }
      }
#pragma unroll
      for (int c = 0; c < NCB; ++c) {
        const int c0 = (cb0 + c) * 8;
        if (row < g.M) {
          if (acc_old) {
            // all eight old values in flight before any store (the stores could alias them)
            double2 o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int col = n0 + c0 + j;
              o[j] = col < g.N ? C[(long long)row + (long long)col * ldc] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              accr[c][j] += o[j].x;
              acci[c][j] += o[j].y;
            }
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int col = n0 + c0 + j;
            if (col < g.N) C[(long long)row + (long long)col * ldc] = make_double2(accr[c][j], acci[c][j]);
          }
          // a phase-1 intermediate read by the next launch as an A operand: its final
          // values also go, sliced, into the A tiles of its view (rows >= M and columns
          // >= N of those tiles stay zero from the arena's initial clearing).  Column
          // chunks past the view's last k-step belong to no tile of this row: writing
          // them would land in the next row tile's tiles.
          if (slice_out && (n0 + c0) / SP_TK < s_nks) {
            double2 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
              v[j] = (n0 + c0 + j) < g.N ? make_double2(accr[c][j], acci[c][j]) : make_double2(0.0, 0.0);
            const int col0 = n0 + c0;
            const long long unit = g.s_off + 2ll * ((long long)job.tm * s_nks + col0 / SP_TK);
            if (unit + 2 <= arenas.units[ARENA_T])
              store_chunk(arenas.a[ARENA_T] + unit * SPLIT_UNIT, A_PLANE, chunk_off(row - m0, (col0 / 8) & 1), v);
          }
        }
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == SP_MMA_WARP) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

cudaError_t launch_grouped_zgemm_split(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms,
                                       Bases bases, SplitArenas arenas, int* fault, long long wait_limit,
                                       int term_alpha, cudaStream_t st) {
  if (njobs <= 0) return cudaSuccess;
  if (!fault || wait_limit < 0) return cudaErrorInvalidValue;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = ensure_smem_attr(grouped_zgemm_split_kernel, SMEM_BYTES, attr);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (nsm <= 0) nsm = 148;
  const int grid = njobs < nsm ? njobs : nsm;
  grouped_zgemm_split_kernel<<<grid, SP_THREADS, SMEM_BYTES, st>>>(jobs, njobs, groups, terms, bases, arenas,
                                                                    fault, wait_limit, term_alpha ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_slice_tiles(const SView* views, const STile* tiles, int ntiles, const double2* in,
                               unsigned char* arena, long long arena_units, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  slice_tiles_kernel<<<ntiles, 256, 0, st>>>(views, tiles, in, arena, arena_units);
  return cudaGetLastError();
}

}  // namespace tsc
