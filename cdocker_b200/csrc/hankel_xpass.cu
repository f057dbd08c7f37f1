// hankel_xpass.cu -- the precision forms' x pass on tcgen05 with the operator resident in
// shared memory (every grid size n in {32, 64, 96, 128}).
//
// For one spectral column c and channel k, the x-direction forward DFT, the conjugate product
// with the receptor spectrum and the inverse DFT collapse into one circulant contraction
//     B(x') = sum_x P~((x + x') mod n) L(x)              (P~: receptor over (y,z) only, x n)
// with real outputs  Re B(x') = sum_x Re P~ Re L + Im P~ Im L
// and  imaginary     Im B(x') = sum_x Im P~ Re L - Re P~ Im L.
// Here the rotations are the MMA's M dimension (128 per tile, one TMEM lane each) and the
// outputs x' its N dimension (N = the tile's largest window, rounded up to 16, so rows that no
// rotation of the tile keeps are never computed). K = 16 per step: the real parts of one
// 8-plane chunk of the ligand (K core matrix 0) and their imaginary parts (core matrix 1).
//
// The operator is a Hankel matrix in (x', x): entry P~(x + x'). For output group i (x' = 8i..
// 8i+7) and K-step j (x = 8j..8j+7) its 8 x 8 core matrix is H[i + j], where
//     H[g][r][d] = P~((8g + r + d) mod n)     (16-byte row r of 8 values d)
// so one buffer of n/8 + jc - 1 such 128-byte groups holds every K-step's tile at once: the
// shared-memory descriptor of K-step j starts at group j and steps 128 bytes per output group
// (SBO = 128). Three buffers per (channel, hi/lo part) -- Re P~, Im P~ and -Re P~ -- give the
// real-output operand (core matrices Re | Im: LBO = one buffer) and the imaginary-output operand
// (Im | -Re). The whole column's operator (all channels, hi and lo) is built once per CTA from
// P~ and stays resident: no operator bytes are streamed per tile.
//
// CTA = COLS columns, persistent over the wave's 128-rotation tiles; 288 threads:
//   warps 0-3  producers. Tiled rows (the default): thread 0 issues per stage (one to three
//              K-steps of one channel, all COLS columns) one tensor copy per K-step and column of
//              the 128 rotations' rows, already in the K-major swizzled layout, completing on the
//              stage's "full" mbarrier by byte count. Untiled rows: thread = rotation of the tile;
//              16-byte cp.async copies of its ligand rows (rows of chunks the rotation does not
//              touch are zero-filled by the copy itself), then one cp.async-completion arrival;
//   warp 4     MMA issuer (one elected lane issues): per K-step and column 2 (real, imaginary) x 2
//              (split-FP16: operator hi, lo) or x 3 (split-BF16: hi*hi, lo*hi, hi*lo) MMAs;
//              commits each stage (1 or 2 K-steps) to its "empty" mbarrier and each tile to a
//              TMEM "full" mbarrier;
//   warps 5-8  epilogue: TMEM -> B of tile t while the MMAs of tile t+1 accumulate into the
//              other of two TMEM accumulator sets (TMEM "empty" mbarrier per set).
// Every wait is bounded; a wait that gives up sets the fault flag, the other roles stop at their
// next wait, issued copies land and TMEM is freed.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>

#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr int HX_R = 128;               // rotations per tile (MMA M)
constexpr int HX_THREADS = 288;         // 9 warps
constexpr int HX_PRODUCERS = 128;       // warps 0-3
constexpr int HX_MMA_WARP = 4;
constexpr int HX_MAXSTAGES = 32;
constexpr int HX_JMAX = 4;              // 8-plane chunks of the ligand box (Lb <= 32)
constexpr uint32_t HX_CORE = 128;       // one 8 x 16-byte core matrix
constexpr uint32_t HX_TILE = 16 * HX_CORE * 2;  // 4 KB: 128 rotations x K 16 (one part)
constexpr long kWaitLimit = 1l << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: K-major, no swizzle (LBO: K direction, SBO: M/N direction)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// shared-memory matrix descriptor: K-major with 32-byte swizzle (rows of 32 bytes = one K-step
// of 16 values, 8-row atoms of 256 bytes; SBO: M/N stride of the atoms; LBO unused: 1)
__device__ __forceinline__ uint64_t make_desc_sw32(uint32_t saddr, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)6 << 61;  // layout type 6: 32-byte swizzle
  return d;
}

// shared-memory matrix descriptor: K-major with 64-byte swizzle (rows of 64 bytes = two K-steps
// of 16 values, 8-row atoms of 512 bytes; SBO: M/N stride of the atoms; LBO unused: 1)
__device__ __forceinline__ uint64_t make_desc_sw64(uint32_t saddr, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;  // layout type 4: 64-byte swizzle
  return d;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int* stop) {
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
    if (i > 32) {
      if (stop && *stop) return false;  // another role gave up: stop waiting
      __nanosleep(40);
    }
  }
  return false;
}

__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "elect.sync _|P, 0xffffffff;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(pred));
  return pred != 0;
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// one 32-byte store (eight floats; p 32-byte aligned)
__device__ __forceinline__ void st_v8(void* p, float a0, float a1, float a2, float a3, float a4, float a5,
                                      float a6, float a7) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a0), "f"(a1), "f"(a2),
               "f"(a3), "f"(a4), "f"(a5), "f"(a6), "f"(a7)
               : "memory");
}

// hi/lo parts of a value (16-bit patterns): split BF16, or split FP16 of a pre-scaled value
template <bool F16>
__device__ __forceinline__ void split16(float v, uint16_t& hi, uint16_t& lo) {
  if constexpr (F16) {
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(__fsub_rn(v, __half2float(h)));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
  } else {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h)));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
  }
}

struct HxScale {
  float s[KMAX];  // split-FP16 form: 2^-sigma_k per channel (the ligand rows carry 2^sigma_k)
};

// The tile's stage plan, read from its first rotation record (k_tile_plan): per active channel
// 4 bits each of channel id, first and last K-step; the stage count, the channel count and the
// largest window of the tile's valid rotations.
struct TilePlan {
  uint64_t pk, pl, ph;
  int nact, steps, wmax;
};

__device__ __forceinline__ TilePlan load_plan(const RotRec* rec0) {
  const uint4* tpv = reinterpret_cast<const uint4*>(rec0->tplan);
  const uint4 t01 = tpv[0], t23 = tpv[1];
  TilePlan p;
  p.pk = ((uint64_t)t01.y << 32) | t01.x;
  p.pl = ((uint64_t)t01.w << 32) | t01.z;
  p.ph = ((uint64_t)t23.y << 32) | t23.x;
  p.nact = (int)(t23.z & 0xFFFFu);
  p.wmax = (int)(t23.z >> 16);
  p.steps = (int)t23.w;
  return p;
}

// N of the tile's MMAs: its largest window rounded up to 16 (M = 128 needs N % 16 == 0)
__device__ __forceinline__ int tile_n(int wmax) { return max(16, (wmax + 15) & ~15); }

template <bool F16>
__device__ __forceinline__ uint32_t make_idesc(int n) {
  // kind::f16: D f32 (bit 4), A/B BF16 (type 1 at bits 7, 10) or FP16 (type 0), both K-major,
  // N >> 3 at bit 17, M >> 4 at bit 24
  return (1u << 4) | (F16 ? 0u : ((1u << 7) | (1u << 10))) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(HX_R >> 4) << 24);
}

// Shared-memory plan of one CTA (bytes), shared by the kernel and its launcher.
struct HxLayout {
  uint32_t S;         // one Hankel buffer: G groups x 128 B
  uint32_t op;        // the column operator: COLS x K x (hi, lo) x 3 buffers
  uint32_t ring;      // offset of the ring: op rounded up to 1 KB (swizzled tiles stay aligned)
  uint32_t ksub;      // one K-step of a stage: COLS x LPARTS x 4 KB
  uint32_t stage;     // one ring stage: ks K-steps
  uint32_t build;     // scratch of the operator build (inside the ring area)
};

__host__ __device__ inline HxLayout hx_layout(int n, int K, int cols, bool f16, int G, int ks) {
  HxLayout L;
  L.S = (uint32_t)G * HX_CORE;
  L.op = (uint32_t)cols * K * 2 * 3 * L.S;
  L.ring = (L.op + 1023u) & ~1023u;
  L.ksub = (uint32_t)cols * (f16 ? 1 : 2) * HX_TILE;
  L.stage = (uint32_t)ks * L.ksub;
  // P~ of the CTA's columns (float2) + their four split arrays (re hi, re lo, im hi, im lo),
  // each n + 32 halves long (the first 32 repeated after the end: no wrap in the group build)
  L.build = (uint32_t)cols * K * n * 8 + (uint32_t)cols * K * 4 * (n + 32) * 2;
  return L;
}

template <int N, int COLS, bool F16>
__global__ void __launch_bounds__(HX_THREADS, 2)
    k_xpass_hankel(const __grid_constant__ CUtensorMap rows_map, WaveArgs a, const float2* __restrict__ pt,
                   HxScale sc, int jc, int G, int nb, int ks, int split) {
  constexpr int NCOL = N * (N / 2 + 1);
  constexpr int LPARTS = F16 ? 1 : 2;
  constexpr int NMAX = N;                          // TMEM columns of one output block (re or im)
  constexpr uint32_t DSET = (uint32_t)COLS * 2 * NMAX;  // one accumulator set
  constexpr uint32_t TCOLS = (2 * DSET <= 32) ? 32 : (2 * DSET <= 64) ? 64 : (2 * DSET <= 128) ? 128
                             : (2 * DSET <= 256) ? 256 : 512;
  static_assert(2 * DSET <= 512, "two accumulator sets fit tensor memory");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t s_full[HX_MAXSTAGES];
  __shared__ __align__(8) uint64_t s_empty[HX_MAXSTAGES];
  __shared__ __align__(8) uint64_t s_tfull[2];
  __shared__ __align__(8) uint64_t s_tempty[2];
  __shared__ volatile int s_fail;
  __shared__ uint32_t s_tmem;
  const int K = a.K;
  const HxLayout L = hx_layout(N, K, COLS, F16, G, ks);
  unsigned char* op = base;              // resident operator
  unsigned char* ring = base + L.ring;   // ring stages (the operator build uses it first)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // CTA = (column group, part): the wave's tiles split into `split` contiguous parts, so that
  // the last round of CTAs is less ragged (each part builds its own operator)
  const int c0 = (int)(blockIdx.x / split) * COLS;
  const int part = (int)(blockIdx.x % split);
  const int ntiles_all = (a.nrot + HX_R - 1) / HX_R;
  const int tbeg = part * ntiles_all / split;
  const int ntiles = (part + 1) * ntiles_all / split;  // one past the CTA's last tile

  if (tid == 0) {
    for (int b = 0; b < nb; ++b) {
      // full: one cp.async arrival per producer thread, or (tiled rows) the one expect_tx arrival
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_full[b])),
                   "r"(a.lop_tiled ? 1 : HX_PRODUCERS));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_empty[b])));
    }
    for (int d = 0; d < 2; ++d) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_tfull[d])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&s_tempty[d])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }

  // ---- operator build: P~ of the CTA's columns -> split arrays -> Hankel groups
  {
    constexpr int NP = N + 32;  // split arrays repeat their first 32 halves after the end
    float2* s_pt = reinterpret_cast<float2*>(ring);                               // [cols][K][N]
    uint16_t* s_sp = reinterpret_cast<uint16_t*>(ring + (size_t)COLS * K * N * 8);  // [cols][K][4][NP]
    for (int i = tid; i < COLS * K * N; i += HX_THREADS) {
      const int cc = i / (K * N), rem = i - cc * K * N;
      s_pt[i] = pt[((size_t)(c0 + cc) * K) * N + rem];
    }
    __syncthreads();
    for (int i = tid; i < COLS * K * NP; i += HX_THREADS) {
      const int ck = i / NP, m = i - ck * NP;
      const int k = ck % K;
      const float scale = F16 ? sc.s[k] : 1.f;
      const float2 v = s_pt[ck * N + (m < N ? m : m - N)];
      uint16_t h, l;
      uint16_t* dst = s_sp + (size_t)ck * 4 * NP + m;
      split16<F16>(F16 ? __fmul_rn(v.x, scale) : v.x, h, l);
      dst[0] = h;
      dst[NP] = l;
      split16<F16>(F16 ? __fmul_rn(v.y, scale) : v.y, h, l);
      dst[2 * NP] = h;
      dst[3 * NP] = l;
    }
    __syncthreads();
    // one 128-byte group per item: [cc][k][hl][buf (Re, Im, -Re)][g] x 8 rows, row r holds
    // P~(8g + r + d), d < 8 -- halves r .. r + 7 of the 16 at 8g: two aligned 16-byte loads,
    // then per row four words picked (r even) or funnel-shifted by one half (r odd); -Re is the
    // negated Re split (sign bits flipped: negation is exact)
    const int groups = COLS * K * 2 * 3 * G;
    for (int i = tid; i < groups; i += HX_THREADS) {
      const int g = i % G;
      const int t = i / G;  // ((cc * K + k) * 2 + hl) * 3 + buf
      const int buf = t % 3, hl = (t / 3) & 1, ck = t / 6;
      const uint16_t* src = s_sp + (size_t)ck * 4 * NP + (size_t)((buf == 1 ? 2 : 0) + hl) * NP + 8 * g;
      const uint4 c0v = *reinterpret_cast<const uint4*>(src);
      const uint4 c1v = *reinterpret_cast<const uint4*>(src + 8);
      const uint32_t W[8] = {c0v.x, c0v.y, c0v.z, c0v.w, c1v.x, c1v.y, c1v.z, c1v.w};
      const uint32_t neg = buf == 2 ? 0x80008000u : 0u;
      uint4* dst = reinterpret_cast<uint4*>(op) + (size_t)i * 8;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
          w[q] = ((r & 1) ? __funnelshift_r(W[r / 2 + q], W[r / 2 + q + 1], 16) : W[r / 2 + q]) ^ neg;
        dst[r] = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    // the groups are read by the tensor cores (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t ring_s = smem_u32(ring);
  const uint32_t op_s = smem_u32(op);

  if (warp < HX_PRODUCERS / 32 && a.lop_tiled) {
    // ---- producer, tiled rows: one thread issues every stage as tensor copies of column c of
    // a row set (128 rotations x one K-step, both parts in split-BF16; rows_map applies the
    // tensor cores' swizzle; untouched chunks already zero); the copies complete on the stage's
    // full barrier by their byte count, in the async proxy the tensor cores read
    if (tid == 0) {
      const uint64_t map = reinterpret_cast<uint64_t>(&rows_map);
      int s = 0, b = 0;
      uint32_t round = 0;
      bool ok = true;
      for (int t = tbeg; t < ntiles && ok; ++t) {
        const TilePlan p = load_plan(a.rec + t * HX_R);
        if (p.steps == 0) continue;
        for (int ai = 0; ai < p.nact && ok; ++ai) {
          const int k = (int)((p.pk >> (4 * ai)) & 15);
          const int jlo = (int)((p.pl >> (4 * ai)) & 15), jhi = (int)((p.ph >> (4 * ai)) & 15);
          for (int j0 = jlo; j0 <= jhi; j0 += ks, ++s) {
            if (s >= nb && !mbar_wait(smem_u32(&s_empty[b]), (round - 1) & 1u, &s_fail)) {
              s_fail = 1;
              ok = false;
              break;
            }
            const uint32_t st = ring_s + (uint32_t)b * L.stage;
            const uint32_t full = smem_u32(&s_full[b]);
            const int jn = min(ks, jhi + 1 - j0);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(
                             (uint32_t)(jn * COLS * LPARTS) * (uint32_t)kLopBlock),
                         "r"(full)
                         : "memory");
            for (int jj = 0; jj < jn; ++jj) {
              const int row0 = ((t * K + k) * 4 + (j0 + jj)) * HX_R;  // the row set's first row
#pragma unroll
              for (int cc = 0; cc < COLS; ++cc) {
                const uint32_t dst = st + (uint32_t)jj * L.ksub + (uint32_t)(cc * LPARTS) * HX_TILE;
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                    " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                    "l"(map), "r"(0), "r"(c0 + cc), "r"(row0), "r"(full)
                    : "memory");
              }
            }
            if (++b == nb) {
              b = 0;
              ++round;
            }
          }
        }
      }
      // every copy issued has landed before the CTA can leave (the last use of each ring slot;
      // earlier uses were consumed before their slot was reissued)
      for (int i = max(0, s - nb); i < s; ++i)
        if (!mbar_wait(smem_u32(&s_full[i % nb]), (uint32_t)(i / nb) & 1u, nullptr)) s_fail = 1;
    }
  } else if (warp < HX_PRODUCERS / 32) {
    // ---- producers
    const int rr = tid;
    const uint32_t row_s = (uint32_t)(rr >> 3) * HX_CORE + (uint32_t)(rr & 7) * 16;
    constexpr size_t RS = (size_t)(NCOL / 4) * 32;  // one ligand row (16 B units)
    constexpr int ROWS = 8 * LPARTS;                // rows per (rotation, channel)
    int s = 0, b = 0;      // stages issued, ring slot of stage s
    uint32_t round = 0;    // s / nb (the ring pass), kept as a counter: no division per stage
    // the next tile's plan and this thread's rotation record are loaded one tile ahead, so
    // their latency hides behind the current tile's copies
    struct Ahead {
      TilePlan p;
      uint4 x[4];  // xlo[16] then xhi[16]
      int valid;
    };
    auto fetch = [&](int t, Ahead& f) {
      const int r0 = t * HX_R;
      const int nr = min(HX_R, a.nrot - r0);
      f.p = load_plan(a.rec + r0);
      const RotRec* rec = a.rec + r0 + min(rr, nr - 1);
      f.valid = rec->valid;
      const uint4* xr = reinterpret_cast<const uint4*>(rec->xlo);
#pragma unroll
      for (int i = 0; i < 4; ++i) f.x[i] = xr[i];
    };
    Ahead nxt;
    if (tbeg < ntiles) fetch(tbeg, nxt);
    for (int t = tbeg; t < ntiles; ++t) {
      const Ahead cur = nxt;
      if (t + 1 < ntiles) fetch(t + 1, nxt);
      const int r0 = t * HX_R;
      const int nr = min(HX_R, a.nrot - r0);
      const TilePlan p = cur.p;
      if (p.steps == 0) continue;
      const bool live = rr < nr && cur.valid;
      // this rotation's chunk range per channel, 8 bits each (0x0F: none)
      uint64_t jr_lo = 0, jr_hi = 0;
      {
        const uint4* v = cur.x;
        const short* lo16 = reinterpret_cast<const short*>(&v[0]);
        const short* hi16 = reinterpret_cast<const short*>(&v[2]);
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          uint64_t e = 0x0F;
          const int lo = live ? lo16[k] : 1, hi = live ? hi16[k] : 0;
          if (k < K && lo <= hi) e = (uint64_t)(min(lo >> 3, jc - 1) | (min(hi >> 3, jc - 1) << 4));
          if (k < 8) jr_lo |= e << (8 * k);
          else jr_hi |= e << (8 * (k - 8));
        }
      }
      const int rg = r0 + (rr < nr ? rr : 0);
      const size_t rot_rows = (size_t)(rg >> 3) * K * ROWS * RS + (size_t)(c0 >> 2) * 32 + (rg & 7) * 4 + (c0 & 3);
      bool ok = true;
      for (int ai = 0; ai < p.nact && ok; ++ai) {
        const int k = (int)((p.pk >> (4 * ai)) & 15);
        const int jlo = (int)((p.pl >> (4 * ai)) & 15), jhi = (int)((p.ph >> (4 * ai)) & 15);
        const unsigned int jr = (unsigned int)(((k < 8 ? jr_lo : jr_hi) >> (8 * (k & 7))) & 255);
        const int jl = (int)(jr & 15), jh = (int)(jr >> 4);
        const uint4* src0 = reinterpret_cast<const uint4*>(a.lop) + rot_rows + (size_t)k * ROWS * RS;
        // a stage: K-steps j0 .. min(j0 + ks, jhi + 1) - 1 of this channel
        for (int j0 = jlo; j0 <= jhi; j0 += ks, ++s) {
          if (s >= nb && !mbar_wait(smem_u32(&s_empty[b]), (round - 1) & 1u, &s_fail)) {
            s_fail = 1;
            ok = false;
            break;
          }
          const uint32_t st = ring_s + (uint32_t)b * L.stage;
          const int jn = min(ks, jhi + 1 - j0);
          for (int jj = 0; jj < jn; ++jj) {
            const int j = j0 + jj;
            const bool have = jl <= j && j <= jh;
#pragma unroll
            for (int cc = 0; cc < COLS; ++cc)
#pragma unroll
              for (int hl = 0; hl < LPARTS; ++hl)
#pragma unroll
                for (int part = 0; part < 2; ++part) {
                  const uint4* src = src0 + (size_t)((hl * 4 + j) * 2 + part) * RS + cc;
                  const uint32_t dst = st + (uint32_t)jj * L.ksub + (uint32_t)(cc * LPARTS + hl) * HX_TILE +
                                       (uint32_t)part * (HX_TILE / 2) + row_s;
                  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(have ? 16 : 0)
                               : "memory");
                }
          }
          asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&s_full[b])) : "memory");
          if (++b == nb) {
            b = 0;
            ++round;
          }
        }
      }
      if (!ok) break;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp == HX_MMA_WARP) {
    // ---- MMA issuer: the whole warp runs the loop (uniform control flow), one elected lane
    // issues each stage's MMAs and its commit. Shared-memory descriptors are built once; the
    // start-address field (bits 0-13) holds the byte address >> 4, so moving a descriptor by a
    // 16-byte aligned byte offset adds offset >> 4 (shared addresses stay below 256 KB: no carry
    // out of the field).
    // ligand rows, slot 0: per-thread copies in the no-swizzle layout (re | im core matrices
    // one half-tile apart), or tiled rows in the 32-byte swizzled layout (re | im in each row)
    const bool tiled = a.lop_tiled != 0;
    // (split-BF16 tiled rows: one 8 KB tile of 64-byte rows, 64-byte swizzle, hi part in the
    // first 32 bytes of each row and lo part in the next)
    const uint64_t dring = !tiled ? make_desc(ring_s, HX_TILE / 2, HX_CORE)
                           : F16  ? make_desc_sw32(ring_s, 256)
                                  : make_desc_sw64(ring_s, 512);
    const uint64_t lo_step = tiled ? 2u : (uint64_t)(HX_TILE >> 4);  // to the lo part
    const uint64_t dop = make_desc(op_s, L.S, HX_CORE);              // operator, group 0
    const uint64_t sS = L.S >> 4;
    int s = 0, u = 0, b = 0;
    uint32_t round = 0;
    bool good = true;
    TilePlan pn{};  // the next tile's plan, loaded one tile ahead
    if (tbeg < ntiles) pn = load_plan(a.rec + tbeg * HX_R);
    for (int t = tbeg; t < ntiles && good; ++t) {
      const TilePlan p = pn;
      if (t + 1 < ntiles) pn = load_plan(a.rec + (t + 1) * HX_R);
      if (p.steps == 0) continue;
      const int d = u & 1;
      if (u >= 2 && !__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_tempty[d]), (uint32_t)((u >> 1) - 1) & 1u, &s_fail))) {
        if (lane == 0) s_fail = 1;
        good = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int nt = tile_n(p.wmax);
      const uint32_t idesc = make_idesc<F16>(nt);
      const uint32_t dset = tmem + (uint32_t)d * DSET;
      uint32_t acc0 = 0u;  // the tile's first K-step starts its accumulators
      for (int ai = 0; ai < p.nact && good; ++ai) {
        const int k = (int)((p.pk >> (4 * ai)) & 15);
        const int jlo = (int)((p.pl >> (4 * ai)) & 15), jhi = (int)((p.ph >> (4 * ai)) & 15);
        const uint64_t dopk = dop + (uint64_t)((k * 2 * 3) * L.S >> 4);
        for (int j0 = jlo; j0 <= jhi; j0 += ks, ++s) {
          if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_full[b]), round & 1u, &s_fail))) {
            if (lane == 0) s_fail = 1;
            good = false;
            break;
          }
          // the producers' cp.async writes (generic proxy) reach the tensor core (async proxy);
          // tensor copies (tiled rows) write in the async proxy already
          if (!tiled) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int jn = min(ks, jhi + 1 - j0);
          const uint64_t aslot = dring + (uint64_t)((b * L.stage) >> 4);
          if (elect_one()) {
            for (int jj = 0; jj < jn; ++jj) {
#pragma unroll
              for (int cc = 0; cc < COLS; ++cc) {
                const uint64_t ahi = aslot + (uint64_t)((jj * L.ksub + cc * LPARTS * HX_TILE) >> 4);
                // Re | Im and Im | -Re operands (one buffer apart), hi then lo part (3 buffers on)
                const uint64_t bre_hi = dopk + (uint64_t)(cc * K * 2 * 3) * sS + (uint64_t)((j0 + jj) * (HX_CORE >> 4));
                const uint32_t dre = dset + (uint32_t)(cc * 2 * NMAX), dim = dre + NMAX;
                umma(dre, ahi, bre_hi, idesc, acc0);
                umma(dim, ahi, bre_hi + sS, idesc, acc0);
                if constexpr (!F16) {
                  const uint64_t alo = ahi + lo_step;
                  umma(dre, alo, bre_hi, idesc, 1u);
                  umma(dim, alo, bre_hi + sS, idesc, 1u);
                }
                umma(dre, ahi, bre_hi + 3 * sS, idesc, 1u);
                umma(dim, ahi, bre_hi + 4 * sS, idesc, 1u);
              }
              acc0 = 1u;
            }
            umma_commit(smem_u32(&s_empty[b]));
          }
          __syncwarp();
          acc0 = 1u;
          if (++b == nb) {
            b = 0;
            ++round;
          }
        }
      }
      if (!good) break;
      if (elect_one()) umma_commit(smem_u32(&s_tfull[d]));
      __syncwarp();
      if (lane == 0 && a.work) {
        // column K-steps, and the issued MMA work in units of 128 x 8 x 16 multiply-adds
        atomicAdd(a.work + 2, (unsigned long long)p.steps * COLS);
        atomicAdd(a.work + 3, (unsigned long long)p.steps * COLS * 2 * (F16 ? 2 : 3) * (nt >> 3));
      }
      ++u;
    }
    // the newest commit completes after every earlier MMA of this warp
    if (lane == 0 && s > 0) {
      // the slot and ring pass of stage s - 1 (one step back from the counters)
      const int bl = b == 0 ? nb - 1 : b - 1;
      const uint32_t rl = b == 0 ? round - 1 : round;
      if (!mbar_wait(smem_u32(&s_empty[bl]), rl & 1u, nullptr)) s_fail = 1;
    }
    __syncwarp();
  } else {
    // ---- epilogue: TMEM lane quarter q = rotations 32 q .. 32 q + 31. A thread holds 16
    // consecutive output planes of its rotation per TMEM load and writes them as runs: with two
    // columns, 32 bytes per plane pair (column-pair groups of G >= 2 planes); with one column
    // and single-column groups (G = 4), 32 bytes per 4 planes. Each store fills whole sectors.
    const int q = warp & 3;
    const int rl = 32 * q + lane;
    // plane groups of the B layout: 1, 2, 4 or 8 (a power of two: masks, no division)
    const int G2 = a.bgroup > 1 ? a.bgroup : 1;
    const int gm = G2 - 1;
    const bool bcol = COLS == 1 && a.bcol != 0;
    int u = 0;
    for (int t = tbeg; t < ntiles; ++t) {
      const int r0 = t * HX_R;
      const int nr = min(HX_R, a.nrot - r0);
      const TilePlan p = load_plan(a.rec + r0);
      if (p.steps == 0) continue;
      // the rotation's window, loaded before the wait for the accumulators
      const RotRec* rec = a.rec + r0 + min(rl, nr - 1);
      const int Wr = (rl < nr && rec->valid) ? rec->W[0] : 0;
      const int d = u & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_tfull[d]), (uint32_t)(u >> 1) & 1u, &s_fail))) {
        if (lane == 0) s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int nt = tile_n(p.wmax);
      float4* rowp = reinterpret_cast<float4*>(a.B + (size_t)(r0 + min(rl, nr - 1)) * N * NCOL);
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)d * DSET;
      for (int x0 = 0; x0 < nt; x0 += 16) {
        float re[COLS][16], im[COLS][16];
#pragma unroll
        for (int cc = 0; cc < COLS; ++cc) {
          tmem_ld16(tbase + (uint32_t)(cc * 2 * NMAX + x0), re[cc]);
          tmem_ld16(tbase + (uint32_t)(cc * 2 * NMAX + NMAX + x0), im[cc]);
        }
        tmem_wait_ld();
        // rows at or past the rotation's window are garbage the inverse (y,z) pass never reads;
        // a run that starts inside the window is written whole (every row < N is in bounds)
        if constexpr (COLS == 2) {
          // column-pair groups: float4 (re, im of columns 2m, 2m + 1) of plane xp at
          // (xp - xp % G) NCOL / 2 + m G + xp % G; planes xp, xp + 1 (xp even) adjacent when G >= 2
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const int xp = x0 + i;
            if (xp < Wr) {
              const size_t f4 = (size_t)(xp & ~gm) * (NCOL / 2) + (size_t)(c0 >> 1) * G2 + (xp & gm);
              if (G2 >= 2) {
                st_v8(rowp + f4, re[0][i], im[0][i], re[1][i], im[1][i], re[0][i + 1], im[0][i + 1],
                      re[1][i + 1], im[1][i + 1]);
              } else {
                rowp[f4] = make_float4(re[0][i], im[0][i], re[1][i], im[1][i]);
                rowp[f4 + NCOL / 2] = make_float4(re[0][i + 1], im[0][i + 1], re[1][i + 1], im[1][i + 1]);
              }
            }
          }
        } else if (bcol && G2 >= 4) {
          // single-column groups: float2 of plane xp at (xp - xp % G) NCOL + c G + xp % G; four
          // planes from xp (a multiple of 4) are one 32-byte run
          float2* row2 = reinterpret_cast<float2*>(rowp);
#pragma unroll
          for (int i = 0; i < 16; i += 4) {
            const int xp = x0 + i;
            if (xp < Wr)
              st_v8(row2 + (size_t)(xp & ~gm) * NCOL + (size_t)c0 * G2 + (xp & gm), re[0][i], im[0][i],
                    re[0][i + 1], im[0][i + 1], re[0][i + 2], im[0][i + 2], re[0][i + 3], im[0][i + 3]);
          }
        } else if (bcol && G2 == 2) {
          // single-column groups of 2 planes: one 16-byte run per plane pair
          float2* row2 = reinterpret_cast<float2*>(rowp);
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const int xp = x0 + i;
            if (xp < Wr)
              *reinterpret_cast<float4*>(row2 + (size_t)xp * NCOL + (size_t)c0 * 2) =
                  make_float4(re[0][i], im[0][i], re[0][i + 1], im[0][i + 1]);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int xp = x0 + i;
            if (xp < Wr) {
              if (bcol) {
                reinterpret_cast<float2*>(rowp)[(size_t)(xp & ~gm) * NCOL + (size_t)c0 * G2 + (xp & gm)] =
                    make_float2(re[0][i], im[0][i]);
              } else {
                const size_t f4 = (size_t)(xp & ~gm) * (NCOL / 2) + (size_t)(c0 >> 1) * G2 + (xp & gm);
                reinterpret_cast<float2*>(rowp + f4)[c0 & 1] = make_float2(re[0][i], im[0][i]);
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&s_tempty[d])) : "memory");
      ++u;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && s_fail) atomicOr(a.fault, 1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
  }
}

// shared memory of one CTA: 227 KB in all, of which the kernel's static barriers and flags
// take 1 KB (ptxas) -- the dynamic part's cap
constexpr size_t kSmemCap = 227 * 1024 - 1024;
constexpr size_t kSmemHalf = 110 * 1024;  // per CTA when two share an SM

// tile parts per column group: the smallest estimated time in rounds of CTAs over the device's
// slots (S CTAs per column group, ceil(groups S / slots) rounds of 1/S of the work each), each
// extra part charged 4 % for its operator build; never more parts than tiles
static int hx_split(int groups, int ntiles, int ctas_per_sm) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
      sms = 148;
  }
  if (const char* e = std::getenv("CDK_HX_SPLIT")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= 8) return std::max(1, std::min(v, ntiles));
  }
  const long slots = (long)sms * std::max(1, ctas_per_sm);
  int best = 1;
  double best_cost = 1e30;
  for (int S = 1; S <= 4 && S <= std::max(1, ntiles); ++S) {
    const double rounds = (double)((groups * (long)S + slots - 1) / slots);
    const double cost = rounds / S * (1.0 + 0.04 * (S - 1));
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = S;
    }
  }
  return best;
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The tensor map of a wave's tiled ligand rows: rows of 16 (split-FP16) or 32 (split-BF16) 16-bit
// values, ncol of them per rotation, 128 rotations per row set and K x 4 row sets per tile; a
// box is column c of 128 consecutive rows (one row set), swizzled as the tensor cores read it.
// L2 promotion to 256-byte requests (a row is 32 or 64 bytes; the neighbouring columns' CTAs read
// the rest of each line): measured 50.2 ms per 1e5 rotations at 64^3 split-FP16 with none or
// 128 bytes, 49.9 with 256 and 91 with 64
cudaError_t rows_tensor_map(CUtensorMap* map, const void* rows, int n, int K, int ntiles, bool f16) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(rows) & 127) || ntiles < 1) return cudaErrorInvalidValue;
  const cuuint64_t ncol = (cuuint64_t)n * (n / 2 + 1);
  const cuuint64_t rb = f16 ? 32 : 64;  // bytes per row
  const cuuint64_t dims[3] = {rb / 2, ncol, (cuuint64_t)ntiles * K * 4 * HX_R};
  const cuuint64_t strides[2] = {rb, ncol * rb};
  const cuuint32_t box[3] = {(cuuint32_t)(rb / 2), 1, (cuuint32_t)HX_R};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<void*>(rows), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, f16 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int N, int COLS, bool F16>
cudaError_t launch_hx(const WaveArgs& a, const float2* pt, const HxScale& sc, int jc, int G, int nb, int ks,
                      size_t smem, int ctas_per_sm, cudaStream_t s) {
  constexpr int NCOL = N * (N / 2 + 1);
  auto kern = k_xpass_hankel<N, COLS, F16>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  const int groups = NCOL / COLS;
  const int ntiles = (a.nrot + HX_R - 1) / HX_R;
  const int split = hx_split(groups, ntiles, ctas_per_sm);
  CUtensorMap map{};
  if (a.lop_tiled) {
    e = rows_tensor_map(&map, a.lop, N, a.K, ntiles, F16);
    if (e != cudaSuccess) return e;
  }
  kern<<<groups * split, HX_THREADS, smem, s>>>(map, a, pt, sc, jc, G, nb, ks, split);
  return cudaGetLastError();
}

}  // namespace

bool tensor_maps_available() { return tensor_map_encoder() != nullptr; }

// Shape of the x pass for (n, K, ligand box, form): columns per CTA, Hankel groups, ring stages
// (each of ks K-steps) and dynamic shared memory. cols_pref: 0 = automatic (1), 1 or 2 = that
// many columns (2 only where the operator of two columns fits); ks_pref: 0 = automatic (2 K-steps per
// stage where the ligand box has several and the ring keeps as many K-steps in flight), 1 or 2.
// Returns false when the operator and a minimal ring do not fit one CTA (large K at large n) or
// the box exceeds 32 planes.
bool hankel_plan(int n, int K, int Lb, bool f16, int cols_pref, HankelPlan* out, int nb_cap, int ks_pref) {
  if (!(n == 32 || n == 64 || n == 96 || n == 128) || K < 1 || K > KMAX || Lb < 1 || Lb > 8 * HX_JMAX)
    return false;
  const int jc = (Lb + 7) / 8;
  const int G = n / 8 + jc - 1;
  // one column per CTA unless two are asked for (two measured 20-35 % slower at 64^3)
  for (int cols : {1, 2}) {
    if (cols_pref ? cols != cols_pref : cols != 1) continue;
    if (cols == 2 && n > 64) continue;  // the tensor memory of two double-buffered columns
    // two CTAs per SM when the tensor memory allows (<= 256 columns each) and the operator
    // leaves room for a ring of at least 8 K-steps; else one CTA with the largest ring
    const bool two = 2 * 2 * cols * n <= 256;
    for (int pass = two ? 0 : 1; pass < 2; ++pass) {
      const size_t cap = (pass == 0 ? kSmemHalf : kSmemCap) - 1024;
      // automatic: 3 K-steps per stage where the box has at least 3 (measured over tiled rows,
      // x pass: split-BF16 4.5 % faster at 128^3; split-FP16 4.5 % at 128^3, and 5 % at 96^3 in
      // both forms), except at n <= 64 in the split-FP16 form (2: 3 measured 1.5 % slower), else
      // 2 where it has several, else 1; fewer where the ring would not keep two CTAs per SM
      // busy otherwise (split-BF16 at 64^3: 1, below)
      const int ks_auto = (jc >= 3 && !(f16 && n <= 64)) ? 3 : jc >= 2 ? 2 : 1;
      for (int ks : {4, 3, 2, 1}) {
        if (ks_pref ? ks != ks_pref : ks > ks_auto) continue;
        const HxLayout L = hx_layout(n, K, cols, f16, G, ks);
        if (cap <= L.ring) continue;
        int nb = (int)std::min<size_t>(HX_MAXSTAGES, (cap - L.ring) / L.stage);
        // two CTAs per SM want 8 K-steps in flight, or at least 4 stages (split-BF16 at 64^3: 5
        // stages of one K-step, x pass 72.0 ms per 1e5 rotations against 88.5 with one CTA per
        // SM and 6 stages of 3 K-steps, 82.7 with two CTAs of 2 stages of 2 K-steps)
        const bool enough = pass == 0 ? (nb * ks >= 8 || (nb >= 4 && nb * ks >= 4)) : nb * ks >= 4;
        if (nb < 2 || !enough || (size_t)nb * L.stage < L.build) continue;
        if (nb_cap > 0 && nb_cap < nb && (size_t)nb_cap * L.stage >= L.build && nb_cap >= 2) nb = nb_cap;
        out->cols = cols;
        out->G = G;
        out->jc = jc;
        out->nb = nb;
        out->ks = ks;
        out->smem = (size_t)L.ring + (size_t)nb * L.stage + 1024;
        // a CTA that takes all 512 tensor-memory columns must have its SM alone: its shared
        // memory then keeps a second CTA out (tcgen05.alloc would otherwise stall it)
        if (pass == 1) out->smem = std::max(out->smem, (size_t)120 * 1024);
        out->ctas_per_sm = pass == 0 ? 2 : 1;
        return true;
      }
    }
  }
  return false;
}

// planes per single-column group: 4 (32-byte runs, the default) or 2 (16-byte runs); the
// environment variable CDK_B_COLGROUP overrides it, for measurement
static int hankel_colgroup() {
  static const int g = [] {
    const char* e = std::getenv("CDK_B_COLGROUP");
    const int v = e ? std::atoi(e) : 4;
    return (v == 2 || v == 4) ? v : 4;
  }();
  return g;
}

void hankel_b_layout(const HankelPlan& p, WaveArgs& a) {
  a.bcol = p.cols == 1 ? 1 : 0;
  a.bgroup = p.cols == 1 ? hankel_colgroup() : stream_bgroup();
}

cudaError_t launch_xpass_hankel(const WaveArgs& a, const float2* pt, const float* f16_scale,
                                const HankelPlan& p, cudaStream_t s) {
  if (!a.lop || !pt || a.K > KMAX) return cudaErrorInvalidValue;
  // the B layout must be the plan's (the inverse (y,z) pass reads what this pass writes)
  if ((a.bcol != 0) != (p.cols == 1) || (a.bcol && a.bgroup != 2 && a.bgroup != 4)) return cudaErrorInvalidValue;
  HxScale sc{};
  for (int k = 0; k < a.K; ++k) sc.s[k] = (a.f16 && f16_scale) ? f16_scale[k] : 1.f;
  // the stage plan of every 128-rotation tile (channels, K-steps, largest window); with tiled
  // rows the plane kernel's launch has computed it already (its zero fill follows the plan)
  if (!a.lop_tiled) {
    cudaError_t e = launch_tile_plan(a, p.jc, s);
    if (e != cudaSuccess) return e;
  }
#define CDK_HX(NN)                                                                               \
  case NN:                                                                                       \
    if (a.f16) return p.cols == 2 ? launch_hx<NN, (NN <= 64 ? 2 : 1), true>(a, pt, sc, p.jc, p.G, p.nb, p.ks, p.smem, p.ctas_per_sm, s) \
                                  : launch_hx<NN, 1, true>(a, pt, sc, p.jc, p.G, p.nb, p.ks, p.smem, p.ctas_per_sm, s);             \
    return p.cols == 2 ? launch_hx<NN, (NN <= 64 ? 2 : 1), false>(a, pt, sc, p.jc, p.G, p.nb, p.ks, p.smem, p.ctas_per_sm, s)       \
                       : launch_hx<NN, 1, false>(a, pt, sc, p.jc, p.G, p.nb, p.ks, p.smem, p.ctas_per_sm, s);
  switch (a.n) {
    CDK_HX(32)
    CDK_HX(64)
    CDK_HX(96)
    CDK_HX(128)
    default:
      return cudaErrorInvalidValue;
  }
#undef CDK_HX
}

}  // namespace cdk
