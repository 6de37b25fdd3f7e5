// MWFJ contraction on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// For one frequency f the multi-window transform is a matrix product
//
//   D[c, n] = sum_k A[c, k] B[k, n]
//     A[c, (i, 0)] = I0_i(f, c)          A[c, (i, 1)] = I1_i(f, c) / k
//     B[(i, 0), n] = g_{i-1, n}(f)       B[(i, 1), n] = b_{i, n}(f)
//
// over the intervals i of the shared pair geometry, with n = 2 w + part the
// real / imaginary part of window w, followed by |D[c, 2w] + i D[c, 2w+1]| /
// k^2 (fj_earthquake's magnitude, src/ccfj-gpu.pyx:282-284) and the
// per-frequency normalisation. A is generated on the fly (the station-
// amortised FP32 special functions, one thread per velocity); B is the
// windows' interval data, prepared once. Both are split into fp16 hi + lo
// parts (22 bits of mantissa per operand) and the product is formed as
// A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32 accumulation in tensor memory
// (FP16x3). fp16's range is kept by exact power-of-two scales: per row
// (velocity) of A from a bound of its entries, per (frequency, window) of B
// from the largest spectrum value, both undone in the epilogue; and the
// slope column uses I1 / (k s) against the spectrum difference g2 - g1
// (s = max(r2 - r1, 0.1), so that (I1 / k) b = (I1 / (k s)) (g2 - g1)).
//
// CTA: 256 threads = 256 velocities (two M = 128 accumulators), one
// frequency, all windows (N = 2 nwin padded to a multiple of 16, <= 256).
// Per chunk of 16 intervals (K = 32): every thread writes its 32 A values
// (hi and lo) into shared memory in the K-major, no-swizzle canonical
// layout; one thread waits for the chunk's B (a 1-D bulk copy, issued two
// chunks ahead), issues 12 tcgen05.mma and commits them to an mbarrier that
// releases the stage. Two stages. All waits are bounded; a wait that runs
// out sets an error flag, drains what is in flight and returns.
#include <cuda_fp16.h>
#include <stdint.h>

#include "fj_cells.cuh"
#include "fj_fft.cuh"

namespace ccfj {

namespace tc {

constexpr int kThreads = 256;       // velocities per CTA (2 x M = 128)
constexpr int kChunkI = 16;         // intervals per chunk
constexpr int kChunkK = 2 * kChunkI;  // K per chunk (I0 and I1/k per interval)
constexpr int kSlices = kChunkK / 16;  // MMA K = 16 for 16-bit operands
constexpr int kSliceBytes128 = 128 * 16 * 2;  // one K-slice of a 128-row operand: 4096 B
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz: a wait longer than this is an error

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false if the phase did not complete within `limit` cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// 1-D bulk copy global -> shared, completion counted on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// K-major, no-swizzle shared-memory matrix descriptor: core matrices of 8
// rows x 16 bytes, LBO = bytes between the two K halves of an MMA K-slice,
// SBO = bytes between 8-row groups; version 1 (tcgen05).
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(p);
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

// Instruction descriptor of kind::f16: F16 A and B (K-major, format 0), F32 D.
__host__ __device__ constexpr uint32_t instr_desc_f16(int M, int N) {
  return (1u << 4)                       // D format F32
         | (0u << 7)                     // A format F16
         | (0u << 10)                    // B format F16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// fp16 hi / lo split of v: hi = rn(v), lo = rn(v - hi).
__device__ __forceinline__ void split_f16(float v, __half& hi, __half& lo) {
  hi = __float2half_rn(v);
  lo = __float2half_rn(v - __half2float(hi));
}

// The same split of two values at once (the two K columns of one interval:
// one packed conversion each for hi and lo, one paired subtraction).
__device__ __forceinline__ void split_f16x2(float a, float b, __half2& hi, __half2& lo) {
  hi = __floats2half2_rn(a, b);
  const float2 h = __half22float2(hi);
  lo = __floats2half2_rn(a - h.x, b - h.y);
}

// 2^(14 - e) for bound = m 2^e (m in [0.5, 1)): a value of magnitude <= bound
// times it stays below 2^14 (fp16 holds up to 65504); 1 for a bound that is
// zero or not finite; the exponent clamped to [-120, 120] (normal floats).
__device__ __forceinline__ float pow2_scale_below_2_14(float bound) {
  if (!(bound > 0.0f) || !isfinite(bound)) return 1.0f;
  int e;
  frexpf(bound, &e);
  return ldexpf(1.0f, max(-120, min(120, 14 - e)));
}

}  // namespace tc

struct MwTcDev {
  const float* rs;
  const uint4* bchunks;     // [nf][nchunks] chunks of (hi, lo) B tiles, chunk_bytes each
  const float* f;
  const float* c;
  const float2* dinv;       // [nr + 1]: (r_i - r_{i-1}, 1 / max(r_i - r_{i-1}, 0.1))
  const float* bounds;      // [2]: max |r|, max |r_i - r_{i-1}| (row scales of A)
  const float* bscale;      // [nwin][nf]: power-of-two scale of B per (window, frequency)
  float* out;               // [nwin][nc][nf]
  unsigned int* err;        // this call's flag: set to 1 when a bounded wait runs out
  unsigned int* sticky;     // process-wide flag (g_mw_tc_error) set alongside, or NULL
  int nr, nf, nc, nwin;
  int N;                    // 2 nwin padded to a multiple of 16
  int nchunks;              // ceil((nr - 1) / kChunkI)
  int tmem_cols;            // power of two >= 2 N
  float tau;
  long long wait_cycles;    // limit of every mbarrier wait (tc::kWaitCycles)
  int self_test_no_copy;    // self-test only: issue no B copy, so the first wait runs out
};

// Shared-memory layout of one CTA (dynamic):
//   A[stage][half m][hi/lo][slice] 128 rows x 16 K fp16   2*2*2*2*4096 = 64 KB
//   B[stage][hi/lo][slice]         N rows x 16 K fp16     2*2*2*(N*32) B
//   barriers, tmem address
struct TcSmem {
  static constexpr int kABytesStage = 2 * 2 * tc::kSlices * tc::kSliceBytes128;
  __host__ __device__ static int b_bytes_stage(int N) { return 2 * tc::kSlices * N * 32; }
  __host__ __device__ static int total(int N) {
    return 2 * kABytesStage + 2 * b_bytes_stage(N) + 64;
  }
};

// Byte offset of element (row, k) inside one 128-row (or N-row) operand
// tile of kSlices K-slices: slice = k / 16, half = (k % 16) / 8.
__device__ __forceinline__ int tile_off(int row, int k, int rows) {
  const int slice = k >> 4, kk = k & 15;
  return slice * rows * 32 + (row >> 3) * 256 + (kk >> 3) * 128 + (row & 7) * 16 + (kk & 7) * 2;
}

// PAIRED: where both stations of two consecutive intervals have x >= 8, the
// two stations are evaluated, and the two intervals' moments formed, with
// paired FP32 instructions (one lane per station); elsewhere, and without
// PAIRED, one interval at a time.
template <bool PAIRED>
__global__ void __launch_bounds__(tc::kThreads, 2) fj_mw_tc_kernel(MwTcDev a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const int fi = blockIdx.y;
  const int c0 = blockIdx.x * tc::kThreads;
  const int ci = min(c0 + tid, a.nc - 1);
  unsigned char* sA = smem;
  unsigned char* sB = smem + 2 * TcSmem::kABytesStage;
  const int bstage = TcSmem::b_bytes_stage(a.N);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 2 * bstage);  // [0,1] B full, [2,3] MMA done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 4);
  __shared__ int abort_flag;

  if (tid == 0) {
    for (int j = 0; j < 4; ++j) tc::mbar_init(bar + j, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  if (tid < 32) {  // warp 0 owns the tensor-memory allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(tmem_slot)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const uint4* bsrc = a.bchunks + (long long)fi * a.nchunks * (bstage / 16);
  // issue B for chunks 0 and 1
  if (tid == 0 && !a.self_test_no_copy) {
    for (int kc = 0; kc < 2 && kc < a.nchunks; ++kc) {
      tc::mbar_expect_tx(bar + kc, bstage);
      tc::bulk_g2s(sB + kc * bstage, bsrc + (long long)kc * (bstage / 16), bstage, bar + kc);
    }
  }

  // per-thread generator state (one velocity)
  Cell<float> cell;
  cell.init(a.f[fi], a.c[ci]);
  const float tau = a.tau;
  ZB<float> Jz{};
  ZB<float> Yz{};
  Station<float> sp;
  float xp = cell.k * __ldg(a.rs);
  float2 dn = __ldg(a.dinv + 1);
  float dr_next = dn.x;
  // this row's scale: |I0| and |I1 / (k s)| are at most max(1, sqrt(k rmax)) k Dmax
  const float row_bound = fmaxf(1.0f, sqrtf(cell.k * __ldg(a.bounds))) * cell.k * __ldg(a.bounds + 1);
  const float sa = tc::pow2_scale_below_2_14(row_bound);
  const float c0s = sa, c1s = sa * cell.inv_k;  // scales of the two A columns (exact: sa = 2^m)
  cell.eval<true, false, true>(__ldg(a.rs), xp, closed_form<float, false>(cell.k * dr_next, xp, tau),
                               Jz, Yz);
  sp = fjs::make_station(xp, Jz);
  bool ln = closed_form<float, false>(cell.k * dr_next, xp, tau);

  const int mh = tid >> 7;      // accumulator (M half)
  const int row = tid & 127;    // row inside it
  const uint32_t idesc = tc::instr_desc_f16(128, a.N);
  int issued_b = a.self_test_no_copy ? 0 : (a.nchunks < 2 ? a.nchunks : 2);  // thread 0's count
  int committed = 0;                             // MMA groups committed (thread 0's count)

  // Every abort decision is taken on abort_flag right after a barrier, so
  // all threads leave the loop together.
  for (int kc = 0; kc < a.nchunks; ++kc) {
    const int s = kc & 1;
    if (kc >= 2) {
      // the MMAs of chunk kc - 2 released this stage
      if (!tc::mbar_wait(bar + 2 + s, ((kc >> 1) - 1) & 1, a.wait_cycles)) atomicOr(&abort_flag, 1);
      __syncthreads();
      if (abort_flag) break;
      if (tid == 0 && !a.self_test_no_copy) {
        tc::mbar_expect_tx(bar + s, bstage);
        tc::bulk_g2s(sB + s * bstage, bsrc + (long long)kc * (bstage / 16), bstage, bar + s);
        ++issued_b;
      }
    }
    // A of this chunk: I0 and I1/k of intervals 1 + 16 kc + j
    unsigned char* aHi = sA + s * TcSmem::kABytesStage + mh * (2 * tc::kSlices * tc::kSliceBytes128);
    unsigned char* aLo = aHi + tc::kSlices * tc::kSliceBytes128;
    // interval i (stations i - 1, i): I0 and I1 / (k s), scaled
    auto one_interval = [&](int i, float& I0, float& I1k) {
      I0 = 0.f;
      I1k = 0.f;
      if (i < a.nr) {
        const float r = __ldg(a.rs + i);
        const float dr = dr_next;
        const float inv_s = dn.y;  // 1 / max(dr, 0.1)
        dn = __ldg(a.dinv + i + 1);
        dr_next = dn.x;
        const float x = cell.k * r;
        const float dx = cell.k * dr;
        const bool lc = ln;
        ln = closed_form<float, false>(cell.k * dr_next, x, tau);
        cell.eval<true, false, true>(r, x, lc || ln, Jz, Yz);
        const Station<float> st = fjs::make_station(x, Jz);
        float I1;
        fjs::interval_moments<float>(sp, st, dx, lc, I0, I1);
        sp = st;
        I0 *= c0s;
        I1k = I1 * c1s * inv_s;
      }
    };
#pragma unroll 1
    for (int j4 = 0; j4 < tc::kChunkI; j4 += 4) {
      __half2 hi[4], lo[4];
#pragma unroll
      for (int jj = 0; jj < 4; jj += 2) {
        const int i = 1 + kc * tc::kChunkI + j4 + jj;
        float2 I0 = make_float2(0.f, 0.f), I1k = make_float2(0.f, 0.f);
        bool done = false;
#if defined(FJS_HAVE_PAIRED)
        if (PAIRED && i + 1 < a.nr) {
          const float2 rr = make_float2(__ldg(a.rs + i), __ldg(a.rs + i + 1));
          const float2 x = fjs::pmul(fjs::psplat(cell.k), rr);
          if (x.x >= 8.0f && x.y >= 8.0f) {
            // intervals i and i + 1; the state then stands after i + 1
            const float2 dn1 = __ldg(a.dinv + i + 1), dn2 = __ldg(a.dinv + i + 2);
            const float2 dx = fjs::pmul(fjs::psplat(cell.k), make_float2(dr_next, dn1.x));
            const float2 inv_s = make_float2(dn.y, dn1.y);
            const bool lc0 = ln;
            const bool lc1 = closed_form<float, false>(cell.k * dn1.x, x.x, tau);
            ln = closed_form<float, false>(cell.k * dn2.x, x.y, tau);
            dn = dn2;
            dr_next = dn2.x;
            float2 p_hi, p_lo;
            p_hi.x = cell.q_hi * rr.x;
            p_lo.x = fmaf(cell.q_lo, rr.x, fmaf(cell.q_hi, rr.x, -p_hi.x));
            p_hi.y = cell.q_hi * rr.y;
            p_lo.y = fmaf(cell.q_lo, rr.y, fmaf(cell.q_hi, rr.y, -p_hi.y));
            fjs::ZB2 J2;
            float2 b2 = make_float2(0.f, 0.f);
            fjs::eval_large_pair_stations_j(x, p_hi, p_lo, lc0 || lc1 || ln, J2, b2);
            const fjs::Station2 st = fjs::make_station_pair(x, J2, b2);
            if (lc0 == lc1) {
              const fjs::Station2 sa{make_float2(sp.h, st.h.x), make_float2(sp.hp, st.hp.x),
                                     make_float2(sp.hpp, st.hpp.x), make_float2(sp.xz1, st.xz1.x),
                                     make_float2(sp.b, st.b.x)};
              float2 I1;
              fjs::interval_moments_pair(sa, st, dx, lc0, I0, I1);
              I1k = fjs::pmul(fjs::pmul(I1, fjs::psplat(c1s)), inv_s);
            } else {
              const Station<float> s0 = fjs::station_lane(st, 0);
              float I1a, I1b;
              fjs::interval_moments<float>(sp, s0, dx.x, lc0, I0.x, I1a);
              fjs::interval_moments<float>(s0, fjs::station_lane(st, 1), dx.y, lc1, I0.y, I1b);
              I1k = fjs::pmul(fjs::pmul(make_float2(I1a, I1b), fjs::psplat(c1s)), inv_s);
            }
            I0 = fjs::pmul(I0, fjs::psplat(c0s));
            sp = fjs::station_lane(st, 1);
            done = true;
          }
        }
#endif
        if (!done) {
          one_interval(i, I0.x, I1k.x);
          one_interval(i + 1, I0.y, I1k.y);
        }
        tc::split_f16x2(I0.x, I1k.x, hi[jj], lo[jj]);
        tc::split_f16x2(I0.y, I1k.y, hi[jj + 1], lo[jj + 1]);
      }
      const int off = tile_off(row, 2 * j4, 128);
      *reinterpret_cast<uint4*>(aHi + off) = *reinterpret_cast<const uint4*>(hi);
      *reinterpret_cast<uint4*>(aLo + off) = *reinterpret_cast<const uint4*>(lo);
    }
    tc::fence_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      if (!tc::mbar_wait(bar + s, (kc >> 1) & 1, a.wait_cycles)) {
        atomicOr(&abort_flag, 1);
      } else {
        unsigned char* bHi = sB + s * bstage;
        unsigned char* bLo = bHi + tc::kSlices * a.N * 32;
        for (int m = 0; m < 2; ++m) {
          unsigned char* ah = sA + s * TcSmem::kABytesStage + m * (2 * tc::kSlices * tc::kSliceBytes128);
          unsigned char* al = ah + tc::kSlices * tc::kSliceBytes128;
          const uint32_t d = tmem + (uint32_t)(m * a.N);  // accumulator m: columns [m N, (m+1) N)
          for (int sl = 0; sl < tc::kSlices; ++sl) {
            const uint64_t dah = tc::smem_desc(ah + sl * tc::kSliceBytes128, 128, 256);
            const uint64_t dal = tc::smem_desc(al + sl * tc::kSliceBytes128, 128, 256);
            const uint64_t dbh = tc::smem_desc(bHi + sl * a.N * 32, 128, 256);
            const uint64_t dbl = tc::smem_desc(bLo + sl * a.N * 32, 128, 256);
            const uint32_t acc0 = (kc > 0 || sl > 0) ? 1u : 0u;
            tc::mma_f16(d, dah, dbh, idesc, acc0);
            tc::mma_f16(d, dah, dbl, idesc, 1u);
            tc::mma_f16(d, dal, dbh, idesc, 1u);
          }
        }
        tc::mma_commit(bar + 2 + s);
        ++committed;
      }
    }
    __syncthreads();
    if (abort_flag) break;
  }

  // Drain: wait for the last committed MMA group (its commit covers every
  // earlier MMA of this thread) and, after an abort, for every B copy still
  // in flight, before reading or freeing anything.
  __shared__ int n_committed, n_issued, drain_fail;
  if (tid == 0) {
    n_committed = committed;
    n_issued = issued_b;
    drain_fail = 0;
  }
  __syncthreads();
  if (n_committed > 0) {
    const int last = n_committed - 1;
    if (!tc::mbar_wait(bar + 2 + (last & 1), (last >> 1) & 1, a.wait_cycles)) atomicOr(&drain_fail, 1);
  }
  if (abort_flag && tid == 0) {
    for (int kc = n_committed; kc < n_issued; ++kc)
      if (!tc::mbar_wait(bar + (kc & 1), (kc >> 1) & 1, a.wait_cycles)) atomicOr(&drain_fail, 1);
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (!abort_flag && !drain_fail && n_committed == a.nchunks) {
    // epilogue: row `row` of accumulator `mh` -> |Re + i Im| / k^2
    const uint32_t tbase = tmem + ((uint32_t)(tid & 96) << 16) + (uint32_t)(mh * a.N);
    const int c = c0 + tid;
    const float inv_sa = 1.0f / sa;  // exact: a power of two
    for (int col = 0; col < a.N; col += 16) {
      float v[16];
      tc::tmem_ld16(tbase + (uint32_t)col, v);
      if (c < a.nc) {
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          const int w = (col + j) >> 1;
          if (w < a.nwin) {
            const float inv_sb = 1.0f / __ldg(a.bscale + (long long)w * a.nf + fi);
            // the scales are powers of two: undoing them is exact
            const float re = v[j] * inv_sa * inv_sb * cell.inv_k2;
            const float im = v[j + 1] * inv_sa * inv_sb * cell.inv_k2;
            a.out[((long long)w * a.nc + c) * a.nf + fi] = sqrtf(re * re + im * im);
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicOr(a.err, 1u);
    if (a.sticky) atomicOr(a.sticky, 1u);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(a.tmem_cols));
  }
}

// The B operand of every (frequency, chunk of 16 intervals): window w's
// interval data of its real (row 2w) and imaginary (row 2w+1) part --
// g_{i-1} and the difference g_i - g_{i-1} (the slope b_i times
// s_i = max(r_i - r_{i-1}, 0.1), src/FJcpu.cpp:259-261; A carries 1 / s_i) --
// times the (window, frequency) scale, split into fp16 hi and lo, in the
// tensor cores' K-major tile layout. One CTA builds the tiles of kPrepF
// consecutive frequencies and one chunk in shared memory -- reading each
// (window, interval) for those frequencies as one 32-byte piece -- then
// stores each frequency's tile contiguously. Rows past the last window and
// intervals past the last pair are zero.
constexpr int kPrepF = 4;
__global__ void __launch_bounds__(256) mw_tc_prep_kernel(const float2* __restrict__ spec, int ntr,
                                                         int nf, int nwin, int N, int nchunks,
                                                         const float* __restrict__ bscale,
                                                         unsigned char* __restrict__ dst) {
  extern __shared__ uint4 tile_u4[];
  unsigned char* tile = reinterpret_cast<unsigned char*>(tile_u4);
  const int kc = blockIdx.x;
  const int f0 = blockIdx.y * kPrepF;
  const long long chunk_bytes = 2LL * tc::kSlices * N * 32;
  const int half = tc::kSlices * N * 32;  // bytes of the hi (or lo) part
  const int nw2 = N / 2;                  // window slots (rows 2w, 2w+1)
  const int items = kPrepF * nw2 * tc::kChunkI;
  // unrolled: several items' spectrum loads in flight per thread
#pragma unroll 4
  for (int t = threadIdx.x; t < items; t += blockDim.x) {
    const int f = t % kPrepF;
    const int w = (t / kPrepF) % nw2;
    const int jj = t / (kPrepF * nw2);
    const int i = 1 + kc * tc::kChunkI + jj;  // interval i: pairs i-1, i
    const int fi = f0 + f;
    float g0r = 0.f, dr = 0.f, g0i = 0.f, di = 0.f;
    if (w < nwin && i < ntr && fi < nf) {
      const float2 cur = spec[((long long)w * ntr + i) * nf + fi];
      const float2 prv = spec[((long long)w * ntr + i - 1) * nf + fi];
      const float sb = bscale[(long long)w * nf + fi];  // a power of two: exact
      g0r = prv.x * sb;
      dr = (cur.x - prv.x) * sb;
      g0i = prv.y * sb;
      di = (cur.y - prv.y) * sb;
    }
    unsigned char* base = tile + (long long)f * chunk_bytes;
    const float g0v[2] = {g0r, g0i}, dv[2] = {dr, di};
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      __half h0, l0, h1, l1;
      tc::split_f16(g0v[part], h0, l0);
      tc::split_f16(dv[part], h1, l1);
      __half2 hh, ll;
      hh.x = h0;
      hh.y = h1;
      ll.x = l0;
      ll.y = l1;
      const int off = tile_off(2 * w + part, 2 * jj, N);
      *reinterpret_cast<__half2*>(base + off) = hh;
      *reinterpret_cast<__half2*>(base + half + off) = ll;
    }
  }
  __syncthreads();
  const int per_f = (int)(chunk_bytes / 16);
  for (int t = threadIdx.x; t < kPrepF * per_f; t += blockDim.x) {
    const int f = t / per_f, q = t % per_f;
    if (f0 + f < nf)
      reinterpret_cast<uint4*>(dst + ((long long)(f0 + f) * nchunks + kc) * chunk_bytes)[q] =
          tile_u4[f * per_f + q];
  }
}

// (r_i - r_{i-1}, 1 / max(r_i - r_{i-1}, 0.1)) per interval from drs.
__global__ void mw_tc_dinv_kernel(const float* __restrict__ drs, int n, float2* __restrict__ dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dinv[i] = make_float2(drs[i], 1.0f / fmaxf(drs[i], 0.1f));
}

// max |r| and max |r_i - r_{i-1}| (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) mw_tc_bounds_kernel(const float* __restrict__ rs,
                                                            const float* __restrict__ drs, int nr,
                                                            float* __restrict__ out) {
  __shared__ float red[2][32];
  float mr = 0.f, md = 0.f;
  for (int i = threadIdx.x; i <= nr; i += blockDim.x) {
    if (i < nr) mr = fmaxf(mr, fabsf(rs[i]));
    md = fmaxf(md, fabsf(drs[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    md = fmaxf(md, __shfl_xor_sync(0xffffffffu, md, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = mr;
    red[1][threadIdx.x >> 5] = md;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    mr = threadIdx.x < (blockDim.x >> 5) ? red[0][threadIdx.x] : 0.f;
    md = threadIdx.x < (blockDim.x >> 5) ? red[1][threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) {
      mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
      md = fmaxf(md, __shfl_xor_sync(0xffffffffu, md, o));
    }
    if (threadIdx.x == 0) {
      out[0] = mr;
      out[1] = md;
    }
  }
}

// Per (window, frequency): the power-of-two scale that keeps the window's
// B entries (spectrum values and differences of neighbours, at most twice
// the largest |Re| or |Im| over the traces) below 2^14.
__global__ void mw_tc_bscale_kernel(const float2* __restrict__ spec, int ntr, int nf,
                                    float* __restrict__ bscale) {
  __shared__ float red[8][33];
  const int fi = blockIdx.x * 32 + threadIdx.x;
  const int w = blockIdx.y;
  float m = 0.f;
  if (fi < nf)
    for (int i = threadIdx.y; i < ntr; i += 8) {
      const float2 v = spec[((long long)w * ntr + i) * nf + fi];
      m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
  red[threadIdx.y][threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.y == 0 && fi < nf) {
    for (int y = 1; y < 8; ++y) m = fmaxf(m, red[y][threadIdx.x]);
    bscale[(long long)w * nf + fi] = tc::pow2_scale_below_2_14(2.0f * m);
  }
}

// Process-wide device flag: set (never cleared by a transform) whenever a
// bounded wait of the tensor-core kernel ran out; ccfj_device_status reads
// and clears it. Each call also has a flag of its own (MwTcDev::err), which
// host-memory calls read, so overlapping calls never clear or inherit each
// other's timeouts.
__device__ unsigned int g_mw_tc_error = 0;

int mwfj_tensor(const ccfj_eq_args& a, const float2* spec, cudaStream_t s, Scratch& sc,
                unsigned int* call_err, bool paired) {
  const int nr = a.ntr, nf = a.nf, nwin = a.nwin;
  CCFJ_REQUIRE(nr >= 2 && nwin >= 1, "MWFJ tensor path: needs nr >= 2 and nwin >= 1");
  int N = 2 * nwin;
  N = (N + 15) / 16 * 16;
  CCFJ_REQUIRE(N <= 256, "MWFJ tensor path: at most 128 windows (got %d)", nwin);
  int cols = 32;
  while (cols < 2 * N) cols <<= 1;
  float* drs = sc.get_n<float>(nr + 1);
  float* wtr = sc.get_n<float>(nr);
  if (!drs || !wtr) return CCFJ_ERR_ALLOC;
  fj_prep_geom_kernel_shared(a.r, nr, drs, wtr, s);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_prep_geom_kernel");
  const int nchunks = (nr - 1 + tc::kChunkI - 1) / tc::kChunkI;
  const long long chunk_bytes = 2LL * tc::kSlices * N * 32;
  unsigned char* bch = static_cast<unsigned char*>(sc.get((size_t)nf * nchunks * chunk_bytes));
  float2* dinv = sc.get_n<float2>(nr + 1);
  float* bounds = sc.get_n<float>(2);
  float* bscale = sc.get_n<float>((size_t)nwin * nf);
  if (!bch || !dinv || !bounds || !bscale) return CCFJ_ERR_ALLOC;
  CCFJ_REQUIRE(nwin <= 65535, "MWFJ tensor path: nwin=%d", nwin);
  mw_tc_dinv_kernel<<<div_up(nr + 1, 256), 256, 0, s>>>(drs, nr + 1, dinv);
  count_launch();
  CCFJ_LAUNCH_CHECK("mw_tc_dinv_kernel");
  mw_tc_bounds_kernel<<<1, 1024, 0, s>>>(a.r, drs, nr, bounds);
  count_launch();
  CCFJ_LAUNCH_CHECK("mw_tc_bounds_kernel");
  mw_tc_bscale_kernel<<<dim3(div_up(nf, 32), nwin), dim3(32, 8), 0, s>>>(spec, nr, nf, bscale);
  count_launch();
  CCFJ_LAUNCH_CHECK("mw_tc_bscale_kernel");
  const size_t prep_smem = (size_t)kPrepF * chunk_bytes;
  CCFJ_CUDA_TRY(cudaFuncSetAttribute(mw_tc_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)prep_smem));
  mw_tc_prep_kernel<<<dim3(nchunks, div_up(nf, kPrepF)), 256, prep_smem, s>>>(
      spec, nr, nf, nwin, N, nchunks, bscale, bch);
  count_launch();
  CCFJ_LAUNCH_CHECK("mw_tc_prep_kernel");
  unsigned int* sticky = nullptr;
  CCFJ_CUDA_TRY(cudaGetSymbolAddress((void**)&sticky, g_mw_tc_error));
  unsigned int* err = call_err ? call_err : sc.get_n<unsigned int>(1);
  if (!err) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned int), s));
  MwTcDev d{};
  d.rs = a.r;
  d.dinv = dinv;
  d.bounds = bounds;
  d.bscale = bscale;
  d.bchunks = reinterpret_cast<const uint4*>(bch);
  d.f = a.f;
  d.c = a.c;
  d.out = a.out;
  d.err = err;
  d.sticky = sticky;
  d.nr = nr;
  d.nf = nf;
  d.nc = a.nc;
  d.nwin = nwin;
  d.N = N;
  d.nchunks = nchunks;
  d.tmem_cols = cols;
  d.tau = a.tau > 0 ? a.tau : kDefaultTau32;
  d.wait_cycles = tc::kWaitCycles;
  d.self_test_no_copy = 0;
  const int smem = TcSmem::total(N);
  auto* kern = paired ? fj_mw_tc_kernel<true> : fj_mw_tc_kernel<false>;
  CCFJ_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  prof_begin(s);
  kern<<<dim3(div_up(a.nc, tc::kThreads), nf), tc::kThreads, smem, s>>>(d);
  prof_end(s);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_mw_tc_kernel");
  if (a.normalize) return normalize_sets(a.out, nwin, a.nc, nf, s);
  return CCFJ_OK;
}

// Self-test of the timeout path: one CTA of the tensor kernel on a tiny
// problem whose B copy is never issued, with a ~1 ms wait limit. The kernel
// must give up, set the error flag, free its tensor memory and return.
int mw_tc_self_test(cudaStream_t s, int* status) {
  Scratch sc(s);
  const int N = 16, nr = 3, cols = 32;
  const float host_r[3] = {1000.f, 2000.f, 3500.f};
  const float host_fc[2] = {0.1f, 1000.f};
  float* r = sc.get_n<float>(nr);
  float* drs = sc.get_n<float>(nr + 1);
  float* fc = sc.get_n<float>(2);
  float* out = sc.get_n<float>(N);
  unsigned char* bch = static_cast<unsigned char*>(sc.get(2 * tc::kSlices * N * 32));
  if (!r || !drs || !fc || !out || !bch) return CCFJ_ERR_ALLOC;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(r, host_r, sizeof(host_r), cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemcpyAsync(fc, host_fc, sizeof(host_fc), cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemsetAsync(bch, 0, 2 * tc::kSlices * N * 32, s));
  float* wtr = sc.get_n<float>(nr);
  unsigned int* err = sc.get_n<unsigned int>(1);
  if (!wtr || !err) return CCFJ_ERR_ALLOC;
  float2* dinv = sc.get_n<float2>(nr + 1);
  float* bounds = sc.get_n<float>(2);
  float* bscale = sc.get_n<float>(1);
  if (!dinv || !bounds || !bscale) return CCFJ_ERR_ALLOC;
  fj_prep_geom_kernel_shared(r, nr, drs, wtr, s);
  mw_tc_dinv_kernel<<<1, 32, 0, s>>>(drs, nr + 1, dinv);
  mw_tc_bounds_kernel<<<1, 1024, 0, s>>>(r, drs, nr, bounds);
  const float one = 1.0f;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(bscale, &one, sizeof(one), cudaMemcpyHostToDevice, s));
  CCFJ_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned int), s));
  MwTcDev d{};
  d.rs = r;
  d.dinv = dinv;
  d.bounds = bounds;
  d.bscale = bscale;
  d.bchunks = reinterpret_cast<const uint4*>(bch);
  d.f = fc;
  d.c = fc + 1;
  d.out = out;
  d.err = err;
  d.sticky = nullptr;  // the self-test's timeout is not a transform's
  d.nr = nr;
  d.nf = 1;
  d.nc = 1;
  d.nwin = 1;
  d.N = N;
  d.nchunks = 1;
  d.tmem_cols = cols;
  d.tau = kDefaultTau32;
  d.wait_cycles = 2000000;  // ~1 ms
  d.self_test_no_copy = 1;
  const int smem = TcSmem::total(N);
  CCFJ_CUDA_TRY(cudaFuncSetAttribute(fj_mw_tc_kernel<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  fj_mw_tc_kernel<true><<<1, tc::kThreads, smem, s>>>(d);
  count_launch();
  CCFJ_LAUNCH_CHECK("fj_mw_tc_kernel (self-test)");
  bool failed = false;
  const int st = mw_tc_call_error(err, s, &failed);
  if (st != CCFJ_OK) return st;
  *status = failed ? CCFJ_ERR_TIMEOUT : CCFJ_OK;
  return CCFJ_OK;
}

int mw_tc_call_error(const unsigned int* err, cudaStream_t s, bool* failed) {
  unsigned int h = 0;
  CCFJ_CUDA_TRY(cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, s));
  CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
  *failed = h != 0;
  return CCFJ_OK;
}

int mw_tc_sticky_error(cudaStream_t s, bool* failed) {
  unsigned int h = 0;
  const unsigned int zero = 0;
  CCFJ_CUDA_TRY(cudaMemcpyFromSymbolAsync(&h, g_mw_tc_error, sizeof(h), 0, cudaMemcpyDeviceToHost, s));
  CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
  if (h) CCFJ_CUDA_TRY(cudaMemcpyToSymbol(g_mw_tc_error, &zero, sizeof(zero)));
  *failed = h != 0;
  return CCFJ_OK;
}

}  // namespace ccfj

CCFJ_API int ccfj_self_test_wait_timeout(void* stream) {
  ccfj::clear_error();
  int status = CCFJ_OK;
  const int st = ccfj::mw_tc_self_test((cudaStream_t)stream, &status);
  if (st != CCFJ_OK) return st;
  if (status != CCFJ_ERR_TIMEOUT)
    return ccfj::set_error(CCFJ_ERR_CUDA, "self-test: the tensor kernel did not report its timeout");
  return CCFJ_OK;
}
