// stream_xpass.cu -- the precision form's x pass with streamed operands (n = 64).
//
// Same contraction as umma_xpass.cu -- per spectral column and channel, the circulant operator
// T = [[Tr, Ti], [Ti, -Tr]] (T(x', x) = P~((x + x') mod n)) times the ligand's x planes, FP32
// accumulation in tensor memory over all channels; split-BF16 form: operator and ligand hi/lo,
// three products; split-FP16 form: operator hi/lo (scaled by 2^-sigma_k), ligand FP16 (scaled
// by 2^sigma_k), two products -- but no operand is built inside the kernel:
//  * the operator tiles are precomputed once per receptor (k_top_build) as the exact shared-
//    memory image of the K-major, no-swizzle layout and arrive by bulk copies (cp.async.bulk
//    with an mbarrier transaction count);
//  * the ligand rows are written split and packed by the plane kernel (k_spread_yz_direct
//    with a lop buffer: per rotation and channel 16 rows [hi, lo][chunk][re, im] of ncol x 16 B,
//    in 512 B blocks of 8 rotations x 4 columns, so the plane kernel writes 64 B runs and the
//    four stages of a column quad read each block whole) and arrive by 16-byte cp.async copies; rows of x chunks that a rotation does not occupy
//    are zero-filled by the copy itself (source size 0, no read).
// K order: step j (16 wide) = group 2j (re part of planes 8j..8j+7) and group 2j+1 (im part).
// Steps outside the chunks any rotation of the tile occupies are neither loaded nor multiplied;
// k_tile_plan computes that plan once per 128-rotation tile, and the search orders its rotations
// so that a tile's rotations touch the same chunks.
//
// CTA = COLS columns x 128 rotations, 256 threads: 2 columns, a 96 KB ring (6 split-BF16 or 8
// split-FP16 stages), 256 TMEM columns and two CTAs per SM for ligand boxes <= 24 planes, else
// 4 columns (32 bytes of B per (rotation, x')), a 192 KB ring (12 or 16 stages), 512 TMEM
// columns, one CTA per SM. A stage is one K-step of one (channel, column): operator hi, lo and
// ligand (hi, lo) tiles of 4 KB, three (two) MMAs; small stages keep many in flight. Warp-specialized: warps 0-3 produce (thread =
// rotation; thread 0 also issues the operator bulk copies), each stage's "full" mbarrier
// completing when every producer's copies
// have landed (cp.async.mbarrier.arrive.noinc) and the operator bytes arrived; one thread of
// warp 4 waits for it, issues the MMAs and commits them to the stage's "empty" mbarrier, which
// the producers wait on before refilling the buffer. All 8 warps run the epilogue. Every wait
// is bounded; a wait that gives up sets the fault flag, lets issued copies land, frees TMEM.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>

#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr int XS_N = 64;
constexpr int XS_NZH = XS_N / 2 + 1;
constexpr int XS_NCOL = XS_N * XS_NZH;
constexpr int XS_R = 128;
constexpr int XS_M = 128;
constexpr int XS_THREADS = 256;
constexpr int XS_PRODUCERS = 128;  // warps 0-3: one producer thread per rotation of the tile
constexpr int XS_MAXSTAGES = 16;
constexpr int XS_JMAX = 4;                          // x chunks of 8 planes (Lb <= 32)
constexpr uint32_t XS_GROUP = (XS_M / 8) * 128;     // 2048 B: one K group of 8 for 128 rows
constexpr uint32_t XS_STEP = 2 * XS_GROUP;          // 4096 B: one K step of 16
constexpr uint32_t XS_TILE = XS_JMAX * XS_STEP;     // 16 KB: 128 rows x 64 K, bf16 (operator image)
constexpr uint32_t XS_SSTAGE = 4 * XS_STEP;         // 16 KB ring stage: T hi, T lo, L hi, L lo
// Two shapes: 2 columns per CTA with a 96 KB ring (two CTAs per SM, so one CTA's epilogue and
// MMA-issue gaps overlap the other's work) when stages are at most 48 KB (ligand box <= 24
// planes), else 4 columns with a 192 KB ring (one CTA per SM).
template <int COLS, bool F16 = false>
struct XsShape {
  static constexpr uint32_t RING = COLS == 2 ? 96 * 1024 : 192 * 1024;
  static constexpr uint32_t TMEM_COLS = COLS * XS_R;
  static constexpr size_t SMEM = (size_t)RING + 1024;
  static constexpr int MIN_BLOCKS = COLS == 2 ? 2 : 1;
  // ring stage: T hi, T lo, L hi, L lo (split-BF16 form) or T hi, T lo, L (split-FP16 form)
  static constexpr int LPARTS = F16 ? 1 : 2;
  static constexpr uint32_t SSTAGE = (2 + LPARTS) * XS_STEP;
  // kind::f16 instruction descriptor: FP32 accumulation, A and B BF16 (type 1) or FP16 (type 0),
  // both K-major, N = 128 rotations, M = 128 operator rows
  static constexpr uint32_t IDESC = (1u << 4) | (F16 ? 0u : (1u << 7) | (1u << 10)) |
                                    ((uint32_t)(XS_R >> 3) << 17) | ((uint32_t)(XS_M >> 4) << 24);
};
constexpr uint32_t XS_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(XS_R >> 3) << 17) |
                              ((uint32_t)(XS_M >> 4) << 24);
constexpr long kWaitLimit = 1l << 22;
static_assert(XS_NCOL % 4 == 0, "column quads tile the half spectrum");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 32) __nanosleep(40);
  }
  return false;
}

// one lane of a converged warp; the MMA warp runs its loop with all 32 lanes so descriptors and
// addresses stay warp-uniform (uniform registers) and only the elected lane issues
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "elect.sync _|P, 0xffffffff;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(pred));
  return pred != 0;
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc,
                                         uint32_t idesc = XS_IDESC) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void bf16_split(float v, uint16_t& hi, uint16_t& lo) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(l);
}

// Operator image: top[((c * K + k) * 2 + hl) * XS_TILE + j * XS_STEP + part * XS_GROUP
//                     + (m >> 3) * 128 + (m & 7) * 16 + d * 2] = hl part of
//   even rows m = 2x':      part 0: Re P~(x + x'),  part 1: Im P~(x + x')   (real output)
//   odd rows m = 2x' + 1:   part 0: Im P~(x + x'),  part 1: -Re P~(x + x')  (imaginary output)
// with x = 8 j + d; real and imaginary outputs of x' land in adjacent TMEM lanes. One thread
// per 16-byte row.
// Split-FP16 form: the same image of hi/lo FP16 parts of P~ 2^-sigma_k (ChanScale.s[k] =
// 2^-sigma_k); the ligand rows carry 2^sigma_k, so P~ fits the FP16 range.
struct ChanScale {
  float s[KMAX];
};

__device__ __forceinline__ void f16_split(float v, uint16_t& hi, uint16_t& lo) {
  const __half h = __float2half_rn(v);
  const __half l = __float2half_rn(__fsub_rn(v, __half2float(h)));
  hi = __half_as_ushort(h);
  lo = __half_as_ushort(l);
}

template <bool F16>
__global__ void __launch_bounds__(256) k_top_build(int K, const float2* __restrict__ pt,
                                                   uint4* __restrict__ top, ChanScale sc) {
  const int c = blockIdx.x, k = blockIdx.y;
  const float scale = F16 ? sc.s[k] : 1.f;
  __shared__ float2 s_p[XS_N];
  if (threadIdx.x < XS_N) s_p[threadIdx.x] = pt[((size_t)c * K + k) * XS_N + threadIdx.x];
  __syncthreads();
  uint4* dst = top + ((size_t)c * K + k) * 2 * (XS_TILE / 16);
  for (int row = threadIdx.x; row < 2 * (int)(XS_TILE / 16); row += blockDim.x) {
    const int hl = row / (XS_TILE / 16);
    const int rem = row - hl * (XS_TILE / 16);
    const int j = rem / (XS_STEP / 16);
    const int part = (rem / (XS_GROUP / 16)) & 1;
    const int m = rem & (XS_M - 1);
    const int xp = m >> 1;            // rows interleaved: 2x' real output, 2x' + 1 imaginary
    const bool imrow = (m & 1) != 0;
    uint16_t e[8];
#pragma unroll
    for (int d = 0; d < 8; ++d) {
      const float2 v = s_p[(8 * j + d + xp) & (XS_N - 1)];
      const float val = imrow ? (part ? -v.x : v.y) : (part ? v.y : v.x);
      uint16_t h, l;
      if (F16) f16_split(__fmul_rn(val, scale), h, l);
      else bf16_split(val, h, l);
      e[d] = hl ? l : h;
    }
    dst[row] = make_uint4((uint32_t)e[0] | ((uint32_t)e[1] << 16), (uint32_t)e[2] | ((uint32_t)e[3] << 16),
                          (uint32_t)e[4] | ((uint32_t)e[5] << 16), (uint32_t)e[6] | ((uint32_t)e[7] << 16));
  }
}

// The stage plan of each 128-rotation tile, once per wave, into the tile's first RotRec: the
// channels any rotation of the tile touches and, per channel, the union of the K-steps (8-plane
// chunks, clamped to the jc chunks of the box) its rotations touch. Every column CTA of the tile
// reads it with one load instead of rebuilding it.
__global__ void __launch_bounds__(XS_R) k_tile_plan(WaveArgs a, int jc) {
  __shared__ int s_jlo[KMAX], s_jhi[KMAX], s_wmax;
  const int tid = threadIdx.x, lane = tid & 31;
  const int r0 = blockIdx.x * XS_R;
  const int nr = min(XS_R, a.nrot - r0);
  const int K = a.K;
  if (tid < KMAX) {
    s_jlo[tid] = XS_JMAX;
    s_jhi[tid] = -1;
  }
  if (tid == 0) s_wmax = 0;
  __syncthreads();
  const RotRec* rec = a.rec + r0 + min(tid, nr - 1);
  const bool live = tid < nr && rec->valid;
  {
    // the largest window of the tile (x' rows any of its rotations keeps)
    const int wm = __reduce_max_sync(0xffffffffu, live ? rec->W[0] : 0);
    if (lane == 0 && wm > 0) atomicMax(&s_wmax, wm);
  }
  for (int k = 0; k < K; ++k) {
    const int lo = live ? rec->xlo[k] : 1, hi = live ? rec->xhi[k] : 0;
    const int jl = lo <= hi ? min(lo >> 3, jc - 1) : 15;
    const int jh = lo <= hi ? min(hi >> 3, jc - 1) : -1;
    const int wl = __reduce_min_sync(0xffffffffu, jl);
    const int wh = __reduce_max_sync(0xffffffffu, jh);
    if (lane == 0) {
      if (wl < 15) atomicMin(&s_jlo[k], wl);
      if (wh >= 0) atomicMax(&s_jhi[k], wh);
    }
  }
  __syncthreads();
  if (tid == 0) {
    uint64_t pk = 0, pl = 0, ph = 0;
    unsigned int n = 0, steps = 0;
    for (int k = 0; k < K; ++k)
      if (s_jlo[k] <= s_jhi[k]) {
        pk |= (uint64_t)k << (4 * n);
        pl |= (uint64_t)s_jlo[k] << (4 * n);
        ph |= (uint64_t)s_jhi[k] << (4 * n);
        steps += (unsigned int)(s_jhi[k] - s_jlo[k] + 1);
        ++n;
      }
    unsigned long long* tp = a.rec[r0].tplan;
    tp[0] = pk;
    tp[1] = pl;
    tp[2] = ph;
    tp[3] = ((unsigned long long)steps << 32) | ((unsigned long long)min(s_wmax, 0xFFFF) << 16) | n;
  }
}

template <int COLS, bool F16>
__global__ void __launch_bounds__(XS_THREADS, XsShape<COLS, F16>::MIN_BLOCKS)
    k_xpass_stream64(WaveArgs a, const unsigned char* __restrict__ top, int jc) {
  using Shape = XsShape<COLS, F16>;
  constexpr uint32_t XS_SSTAGE = Shape::SSTAGE;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // keep the ring 1024-aligned whatever the dynamic base
  unsigned char* ring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t s_full[XS_MAXSTAGES];
  __shared__ __align__(8) uint64_t s_empty[XS_MAXSTAGES];
  __shared__ int s_fail;
  __shared__ int s_issued, s_consumed;
  __shared__ uint32_t s_tmem;
  __shared__ int s_W[XS_R];
  const int K = a.K;
  // ring: stages of one K-step (operator hi, lo and ligand hi, lo tiles of 4 KB), as many as fit
  const int nb = min(XS_MAXSTAGES, (int)(Shape::RING / XS_SSTAGE));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = blockIdx.x * XS_R;
  const int c0 = blockIdx.y * COLS;
  const int nr = min(XS_R, a.nrot - r0);
  if (tid == 0) {
    for (int b = 0; b < nb; ++b) {
      // full: one cp.async arrival per producer thread + the operator copies' expect_tx arrival
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_full[b])), "r"(XS_PRODUCERS + 1));
      // empty: the MMA thread's tcgen05.commit
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_empty[b])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(Shape::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  // the tile's stage plan (k_tile_plan), one 32-byte load; per active channel 4 bits each of
  // channel id, first and last K-step, so the loops below read no shared memory but the
  // mbarriers
  const uint4* tpv = reinterpret_cast<const uint4*>(a.rec[r0].tplan);
  const uint4 t01 = tpv[0], t23 = tpv[1];
  const uint64_t pk = ((uint64_t)t01.y << 32) | t01.x;
  const uint64_t pl = ((uint64_t)t01.w << 32) | t01.z;
  const uint64_t ph = ((uint64_t)t23.y << 32) | t23.x;
  const int nact = (int)(t23.z & 0xFFFFu);
  const int NS = COLS * (int)t23.w;  // stages: one K-step of one (channel, column)
  // this thread's rotation: its window (epilogue) and, for the producers, its chunk range per
  // channel (8 bits each: jlo | jhi << 4, 0x0F when empty) from one vector load of the record
  uint64_t jr_lo = 0, jr_hi = 0;
  if (tid < XS_R) {
    const RotRec* rec = a.rec + r0 + min(tid, nr - 1);
    const bool live = tid < nr && rec->valid;
    s_W[tid] = live ? rec->W[0] : 0;
    static_assert(KMAX == 16, "x ranges are two 32-byte vectors");
    uint4 v[4];
    const uint4* xr = reinterpret_cast<const uint4*>(rec->xlo);  // xlo[16] then xhi[16]
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = xr[i];
    const short* lo16 = reinterpret_cast<const short*>(&v[0]);
    const short* hi16 = reinterpret_cast<const short*>(&v[2]);
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      uint64_t e = 0x0F;
      const int lo = live ? lo16[k] : 1, hi = live ? hi16[k] : 0;
      // valid rotations keep every plane inside the planned box; the clamp only keeps
      // shared-memory offsets in range whatever the record says
      if (k < K && lo <= hi) e = (uint64_t)(min(lo >> 3, jc - 1) | (min(hi >> 3, jc - 1) << 4));
      if (k < 8) jr_lo |= e << (8 * k);
      else jr_hi |= e << (8 * (k - 8));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const unsigned char* lop = a.lop;
  const uint32_t ring_s = smem_u32(ring);

  if (tid < XS_PRODUCERS) {
    // ---- producers: thread = rotation rr of the tile; per stage its 4 split rows
    const int rr = tid;
    const uint32_t row_s = (uint32_t)(rr >> 3) * 128 + (uint32_t)(rr & 7) * 16;
    const int rg = r0 + (rr < nr ? rr : 0);
    // 16 B units: (((r/8 * K + k) * ROWS + row) * ncol/4 + c/4) * 32 + (r%8) * 4 + c%4 with
    // ROWS = 16 split-BF16 rows [hi, lo][chunk][re, im] or 8 FP16 rows [chunk][re, im]
    constexpr size_t RS = (size_t)(XS_NCOL / 4) * 32;
    constexpr int ROWS = 8 * Shape::LPARTS;
    const size_t rot_rows = (size_t)(rg >> 3) * K * ROWS * RS + (size_t)(c0 >> 2) * 32 + (rg & 7) * 4 + (c0 & 3);
    int s = 0, b = 0;
    uint32_t round = 0;  // s / nb
    for (int ai = 0; ai < nact && s >= 0; ++ai) {
      const int k = (int)((pk >> (4 * ai)) & 15);
      const int jlo = (int)((pl >> (4 * ai)) & 15), jhi = (int)((ph >> (4 * ai)) & 15);
      const unsigned int jr = (unsigned int)(((k < 8 ? jr_lo : jr_hi) >> (8 * (k & 7))) & 255);
      const int jl = (int)(jr & 15), jh = (int)(jr >> 4);
      for (int c = 0; c < COLS && s >= 0; ++c) {
        const uint4* src0 = reinterpret_cast<const uint4*>(lop) + rot_rows + (size_t)k * ROWS * RS + c;
        const unsigned char* tsrc = top + ((size_t)(c0 + c) * K + k) * 2 * XS_TILE;
        for (int j = jlo; j <= jhi; ++j, ++s) {
          if (s >= nb) {
            // the MMAs of stage s - nb must be done with this buffer
            if (!mbar_wait(smem_u32(&s_empty[b]), (round - 1) & 1u)) {
              atomicOr(&s_fail, 1);
              s = -1;
              break;
            }
          }
          const uint32_t st = ring_s + (uint32_t)b * XS_SSTAGE;
          const uint32_t full = smem_u32(&s_full[b]);
          if (tid == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(2 * XS_STEP), "r"(full)
                         : "memory");
#pragma unroll
            for (int hl = 0; hl < 2; ++hl)
              asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                               st + (uint32_t)hl * XS_STEP),
                           "l"(tsrc + (size_t)hl * XS_TILE + (size_t)j * XS_STEP), "r"(XS_STEP), "r"(full)
                           : "memory");
            s_issued = s + 1;
          }
          const bool have = jl <= j && j <= jh;
#pragma unroll
          for (int hl = 0; hl < Shape::LPARTS; ++hl)
#pragma unroll
            for (int part = 0; part < 2; ++part) {
              const uint4* src = src0 + (size_t)((hl * 4 + j) * 2 + part) * RS;
              const uint32_t dst = st + (uint32_t)(2 + hl) * XS_STEP + (uint32_t)part * XS_GROUP + row_s;
              asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(have ? 16 : 0)
                           : "memory");
            }
          asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(full) : "memory");
          if (++b == nb) {
            b = 0;
            ++round;
          }
        }
      }
    }
  } else if (warp == XS_PRODUCERS / 32) {
    // ---- MMA issuer: the whole warp runs the loop, one elected lane issues
    const uint64_t desc0 = make_desc(ring_s, XS_GROUP, 128);
    constexpr uint64_t TU = XS_STEP >> 4;  // one 4 KB tile in descriptor address units
    int s = 0, b = 0;
    uint32_t round = 0;
    bool good = true;
    for (int ai = 0; ai < nact && good; ++ai) {
      const int jlo = (int)((pl >> (4 * ai)) & 15), jhi = (int)((ph >> (4 * ai)) & 15);
      for (int c = 0; c < COLS && good; ++c) {
        const uint32_t d = tmem + (uint32_t)(c * XS_R);
        for (int j = jlo; j <= jhi; ++j, ++s) {
          if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_full[b]), round & 1u))) {
            if (lane == 0) atomicOr(&s_fail, 1);
            good = false;
            break;
          }
          // the producers' cp.async writes (generic proxy) reach the tensor core (async proxy)
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t ah = desc0 + (uint64_t)b * (XS_SSTAGE >> 4);
          const uint32_t acc = (ai > 0 || j > jlo) ? 1u : 0u;  // first product of column c
          // T_hi L_hi, T_hi L_lo, T_lo L_hi (split BF16) or T_hi L, T_lo L (split FP16)
          if (elect_one()) umma_f16(d, ah, ah + 2 * TU, acc, Shape::IDESC);
          if (!F16 && elect_one()) umma_f16(d, ah, ah + 3 * TU, 1u, Shape::IDESC);
          if (elect_one()) umma_f16(d, ah + TU, ah + 2 * TU, 1u, Shape::IDESC);
          if (elect_one())
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&s_empty[b]))
                         : "memory");
          __syncwarp();
          if (++b == nb) {
            b = 0;
            ++round;
          }
        }
      }
    }
    if (lane == 0) {
      s_consumed = s;
      if (s && a.work) atomicAdd(a.work + 2, (unsigned long long)s);  // K-steps issued
      // the newest commit completes after every earlier MMA of this warp
      if (s > 0 && !mbar_wait(smem_u32(&s_empty[(s - 1) % nb]), (uint32_t)((s - 1) / nb) & 1u))
        atomicOr(&s_fail, 1);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  bool ok = s_fail == 0;
  if (!ok && tid == 0) {
    // operator copies issued for stages the MMA thread never consumed: let them land
    for (int t = s_consumed; t < s_issued; ++t)
      mbar_wait(smem_u32(&s_full[t % nb]), (uint32_t)(t / nb) & 1u);
  }
  __syncthreads();
  if (!ok) {
    if (tid == 0) atomicOr(a.fault, 1);
  } else if (NS > 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // ---- epilogue, TMEM -> B without a shared-memory round trip: warp w reads lanes
    // 32 (w % 4) .. + 31 (x' = 16 (w % 4) .. + 15, real and imaginary in adjacent lanes) for
    // the rotation chunks of its half. Lanes 2j and 2j + 1 hold x' = 16 (w % 4) + j; per step
    // of two rotations the even lane writes rotation t and the odd lane rotation t + 1, each
    // taking its missing half from the other through one shuffle: (re, im) of all the CTA's
    // columns for one (rotation, x'), 16 or 32 B
    const int q = warp & 3;
    const int xp = 16 * q + (lane >> 1);
    const int odd = lane & 1;
    // grouped B layout: the lanes' planes x' = 16 q .. 16 q + 15 fill G-plane blocks of 16 G
    // contiguous bytes per column pair (whole sectors for G >= 2)
    const int G = a.bgroup > 1 ? a.bgroup : 1;
    const size_t xoff = (size_t)(xp - xp % G) * (XS_NCOL / 2) + xp % G;  // in float4 units
    for (int jr = 2 * (warp >> 2); jr < 2 * (warp >> 2) + 2; ++jr) {
      float v[COLS][32];
#pragma unroll
      for (int c = 0; c < COLS; ++c)
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(c * XS_R + 32 * jr), v[c]);
#pragma unroll
      for (int t = 0; t < 32; t += 2) {
        float re[COLS], im[COLS];
#pragma unroll
        for (int c = 0; c < COLS; ++c) {
          // even lane: its re of rotation t, the odd lane's im of t; odd lane: the even lane's
          // re of t + 1, its im of t + 1
          const float other = __shfl_xor_sync(0xffffffffu, odd ? v[c][t] : v[c][t + 1], 1);
          re[c] = odd ? other : v[c][t];
          im[c] = odd ? v[c][t + 1] : other;
        }
        const int rr = 32 * jr + t + odd;
        if (rr < nr && xp < s_W[rr]) {
          float4* dst = reinterpret_cast<float4*>(a.B + (size_t)(r0 + rr) * XS_N * XS_NCOL) + xoff + (size_t)(c0 / 2) * G;
#pragma unroll
          for (int c = 0; c < COLS; c += 2) dst[(size_t)(c / 2) * G] = make_float4(re[c], im[c], re[c + 1], im[c + 1]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Shape::TMEM_COLS));
  }
}


}  // namespace

int stream_bgroup() {
  static const int g = [] {
    const char* e = std::getenv("CDK_B_GROUP");
    const int v = e ? std::atoi(e) : 2;
    return (v == 1 || v == 2 || v == 4 || v == 8) ? v : 2;
  }();
  return g;
}

cudaError_t launch_tile_plan(const WaveArgs& a, int jc, cudaStream_t s) {
  if (jc < 1 || jc > XS_JMAX) return cudaErrorInvalidValue;
  k_tile_plan<<<(a.nrot + XS_R - 1) / XS_R, XS_R, 0, s>>>(a, jc);
  return cudaGetLastError();
}

bool stream_supported(int n, int Lb) { return n == 64 && Lb >= 1 && Lb <= 8 * XS_JMAX; }

size_t stream_top_bytes(int n, int K) {
  return n == 64 ? (size_t)XS_NCOL * K * 2 * XS_TILE : 0;
}

size_t stream_lop_bytes_per_rotation(int n, int K, bool f16) {
  // per channel 16 split-BF16 rows or 8 FP16 rows of the half spectrum, 16 B per column
  return (size_t)K * n * (n / 2 + 1) * (f16 ? 128 : 256);
}

cudaError_t launch_top_build(int n, int K, const float2* pt, void* top, const float* f16_scale,
                             cudaStream_t s) {
  if (n != 64 || K > KMAX) return cudaErrorInvalidValue;
  ChanScale sc{};
  for (int k = 0; k < K; ++k) sc.s[k] = f16_scale ? f16_scale[k] : 1.f;
  if (f16_scale) k_top_build<true><<<dim3(XS_NCOL, K), 256, 0, s>>>(K, pt, reinterpret_cast<uint4*>(top), sc);
  else k_top_build<false><<<dim3(XS_NCOL, K), 256, 0, s>>>(K, pt, reinterpret_cast<uint4*>(top), sc);
  return cudaGetLastError();
}

template <int COLS, bool F16>
cudaError_t launch_stream_cols(const WaveArgs& a, const void* top, int jc, cudaStream_t s) {
  using Shape = XsShape<COLS, F16>;
  cudaError_t e = cudaFuncSetAttribute(k_xpass_stream64<COLS, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Shape::SMEM);
  if (e != cudaSuccess) return e;
  // all of the unified L1 as shared memory, so two 2-column CTAs fit one SM
  e = cudaFuncSetAttribute(k_xpass_stream64<COLS, F16>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  dim3 grid((a.nrot + XS_R - 1) / XS_R, XS_NCOL / COLS);
  k_xpass_stream64<COLS, F16><<<grid, XS_THREADS, Shape::SMEM, s>>>(a, reinterpret_cast<const unsigned char*>(top), jc);
  return cudaGetLastError();
}

cudaError_t launch_xpass_stream(const WaveArgs& a, const void* top, cudaStream_t s) {
  if (!stream_supported(a.n, a.Lb) || !a.lop || !top) return cudaErrorInvalidValue;
  const int jc = (a.Lb + 7) / 8;  // K-steps a valid rotation can touch
  // ligand boxes of up to 24 planes: 2 columns, two CTAs per SM; larger boxes: 4 columns
  cudaError_t e = launch_tile_plan(a, jc, s);
  if (e != cudaSuccess) return e;
  if (a.f16) {
    return jc <= 3 ? launch_stream_cols<2, true>(a, top, jc, s) : launch_stream_cols<4, true>(a, top, jc, s);
  }
  return jc <= 3 ? launch_stream_cols<2, false>(a, top, jc, s) : launch_stream_cols<4, false>(a, top, jc, s);
}

}  // namespace cdk
