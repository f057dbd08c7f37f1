// cdk_internal.h -- device data layout and launch interface shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace cdk {

constexpr int KMAX = 16;  // most receptor grids one context can hold

// One conformer's atoms: coords at coord_off (atoms), per-atom parameters at param_off.
struct ConfDesc {
  int coord_off;
  int param_off;
  int n_atoms;
  int pad;
};

// One rotation of the search: unit quaternion (w,x,y,z), its conformer, the output slot.
struct RotDesc {
  float q[4];
  int conf;
  int out;
  int pad0, pad1;
};

// Per-atom ligand parameters: sqrt(epsilon) as FillLigandGrid weighs vdW grids
// (src/FillLigandGrid.cpp:43), the charge (elec grid, :97), and the atom's vdW slot.
struct AtomParam {
  float w_vdw;
  float charge;
  int slot;
  int pad;
};

// Per-rotation record written by the prep kernel.
struct RotRec {
  float mn[3];      // min corner of the rotated ligand (GetMinCoors)
  int W[3];         // translation window per axis: n - int(len/h) - 2
  int ext[3];       // cells touched by the spread per axis (max cell index + 2)
  int valid;        // 1 when every window is non-empty
  int err;          // nonzero when the ligand box exceeded the planned box
  int nA;           // atoms
  short xlo[KMAX];  // per channel: first and last x plane touched (xlo > xhi: empty)
  short xhi[KMAX];
  // streamed tensor-core x pass, first record of each 128-rotation tile only: the tile's stage
  // plan (4 bits per active channel: id, first and last K-step; then active channels and K-steps
  // per column), written by k_tile_plan
  unsigned long long tplan[4];
};
// the x ranges are read as 16-byte vectors
static_assert(offsetof(RotRec, xlo) % 16 == 0 && offsetof(RotRec, tplan) % 16 == 0 && sizeof(RotRec) % 16 == 0,
              "RotRec vector alignment");

// Everything one wave of rotations needs on the device.
struct WaveArgs {
  int n;             // grid edge (cubic)
  int K;             // channels (vdW grids + elec)
  int Lb;            // planned ligand box edge (x planes stored per channel)
  float spacing;
  int nrot;          // rotations in this wave
  int max_atoms;     // stride of rotated-atom storage
  int atom_cap;      // largest ligand of this wave (sizes the direct plane kernel)
  const float* coords;       // [atoms][3]
  const AtomParam* params;   // [atom params]
  const ConfDesc* confs;
  const RotDesc* rots;       // [nrot]
  float4* rot_xyz;           // [nrot][max_atoms]
  RotRec* rec;               // [nrot]
  float2* A;                 // [nrot][K][Lb][ncol]
  float2* B;                 // [nrot][n][ncol], or with bgroup G > 1 [nrot][n/G][ncol/2][G][2]:
                             // the x planes grouped by G, 16 B (two columns) per (plane, pair);
                             // or with bcol [nrot][n/G][ncol][G]: G planes of one column
  int bgroup;                // 0 or 1: plain B layout; 2, 4, 8: grouped (tensor-core x passes)
  int bcol;                  // 1: the grouped layout keeps single columns (G x 8 B runs), for
                             // x passes that own one column per CTA
  int yz_block_stages;       // inverse (y,z) kernel: 0 by grid size (block stages at n <= 64,
                             // octets at n >= 96), 1 block stages, 2 octets
  unsigned long long* keys;  // [nrot]
  unsigned long long* keys2; // precision forms' near-tie break: [nrot][n][2] the two smallest
                             // keys of every window plane (null: not kept)
  const float2* phat;        // [n][K][ncol] (kx position-major)
  const float2* tw;          // [n]
  float* minE;               // output base (indexed by RotDesc.out)
  int* idx;
  int* err_count;
  unsigned long long* work;  // work counters: [0] x planes spread, [1] window planes,
                             // [2] tensor-core column K-steps, [3] MMA units, [4] near-tie
                             // re-scores, [5] near-tie translations changed
  int col_tile;
  int chunk;                 // rotations per CTA in the x pass (0 = default)
  int* fault;                // set when a bounded device wait gave up
  const int* kyof;           // [n] natural frequency at each digit-reversed position; when set
                             // (and ligands have <= 96 atoms) planes are evaluated directly
  int f16;                   // split-FP16 form: the plane kernel writes FP16 rows (8 per rotation
                             // and channel: [chunk][re, im]) of the planes times lscale[k]
  float lscale[KMAX];        // split-FP16 form: 2^sigma_k per channel (a power of two, exact)
  int* range_err;            // split-FP16 form: set when a scaled ligand value left the FP16 range
  unsigned char* lop;        // when set (direct planes): the plane kernel writes the ligand as
                             // split-BF16 or FP16 x-chunk rows here instead of A, in one of
                             // two layouts (lop_tiled)
  int lop_tiled;             // 0: [nrot/8][K][hi/lo][chunk j < 4][re/im][ncol/4][nrot%8][ncol%4]
                             //    x 16 B of 8 planes (nrot rounded up to a multiple of 8), the
                             //    streamed-tile x pass's rows;
                             // 1: 128-rotation row sets [nrot/128][K][chunk j < 4][rotation
                             //    m < 128][ncol] of one row per (rotation, column): 32 B
                             //    [re | im] (split-FP16) or 64 B [hi re | hi im | lo re | lo im]
                             //    (split-BF16) of 8 planes, natural order; the Hankel x pass
                             //    loads column c of a row set (128 rows) with one tensor copy
                             //    per K-step, which applies the tensor cores' 32- or 64-byte
                             //    swizzle; chunks of the tile's stage plan that a valid rotation
                             //    does not touch hold zeros (the plane kernel runs after
                             //    k_tile_plan)
  int plane_rot_major;       // set by the plane kernel's launcher: grid (nrot, K) instead of
                             // (K, nrot)
};
// rotations per tensor-core tile (the MMA's M), and the bytes of one K-step (128 rows of 32 B)
// of one column and part in the tiled ligand-row layout
constexpr int kTileRot = 128;
constexpr size_t kLopBlock = 4096;
// rotations a wave's ligand rows are allocated for
inline size_t lop_rotations(long nrot, bool tiled) {
  return tiled ? (size_t)((nrot + kTileRot - 1) / kTileRot) * kTileRot : (size_t)((nrot + 7) & ~7L);
}
// The automatic tensor-core x pass (variant: opts.reserved[3] = 0) is the Hankel kernel at every
// n; the 64^3 kernel with streamed operator tiles runs on request (3)
inline bool use_stream_tiles(int variant) { return variant == 3; }
// The Hankel x pass loads tiled rows (one tensor copy per K-step and column) unless
// opts.reserved[5] bit 5 asks for per-rotation copies by its producer threads (bit 6, tiled
// rows, is the default). Measured per search against per-rotation copies: 64^3 -13 % (split-FP16)
// and -19 % (split-BF16), 96^3 -6 % and -13 %, 128^3 -3 % and -6 %
// (and the driver provides the tensor-map encoder; without it the per-rotation copies run)
bool tensor_maps_available();
inline bool hankel_tiled(int reserved5) { return !(reserved5 & 32) && tensor_maps_available(); }
// bytes of a wave's ligand rows (per-rotation bytes times the rotations allocated)
inline size_t lop_wave_bytes(long nrot, bool tiled, size_t per_rotation) {
  return lop_rotations(nrot, tiled) * per_rotation;
}

// Launchers (stream-ordered, no synchronisation). Return cudaError_t of the launch.
cudaError_t launch_prep(const WaveArgs& a, cudaStream_t s);
// A wave's lowest-energy pose with its FP64 re-score (precision forms, per wave).
constexpr int kTopMax = 32;
struct TopPose {
  int out;     // the rotation's output slot (RotDesc.out); -1: unused
  int lin;     // kept translation, linear index (x * n + y) * n + z
  float e;     // the search's energy there
  int pad;
  double e64;  // its FP64 direct grid-energy sum
};
cudaError_t launch_topk_rescore(const WaveArgs& a, const float* grids, int k, TopPose* out, cudaStream_t s);
// FP64 near-tie break of the argmin over the planes' two smallest keys (a.keys2), before
// launch_finalize; grids: the receptor grids [K][n][n][n]
cudaError_t launch_tiebreak(const WaveArgs& a, const float* grids, float tol, cudaStream_t s);
// rotation grouping for the tensor-core x pass (a stable counting sort of the rotation list on
// which channels reach the ligand box's last 8-plane chunk); scratch of group_rotations_bytes
size_t group_rotations_bytes(long nrot);
cudaError_t launch_group_rotations(const RotDesc* rots, const ConfDesc* confs, const float* coords,
                                   const AtomParam* params, long nrot, int max_atoms, int K, float h,
                                   int jc, void* scratch, RotDesc** sorted, cudaStream_t s);
cudaError_t launch_spread_yz(const WaveArgs& a, cudaStream_t s);
cudaError_t launch_xpass(const WaveArgs& a, cudaStream_t s);
cudaError_t launch_yz_inv_argmin(const WaveArgs& a, cudaStream_t s);
cudaError_t launch_finalize(const WaveArgs& a, cudaStream_t s);
// Finalize for waves whose rotations belong to different requests: minE goes to
// ebase[RotDesc.out], the three indices to ibase[RotDesc.pad0 .. +2].
cudaError_t launch_finalize_server(const WaveArgs& a, float* ebase, int* ibase, cudaStream_t s);
// Dense forward transform of K receptor grids [K][n][n][n] -> phat [n][K][ncol].
cudaError_t launch_receptor_fft(int n, int K, const float* grids, float2* scratch,
                                float2* phat, const float2* tw, int col_tile, cudaStream_t s);
// Shared memory per CTA of the FP32 x pass for given n, K, column tile.
size_t xpass2_smem_bytes(int n, int K, int col_tile);
int pick_col_tile(int n, int K);
// Dense FillLigandGrid on the GPU.
cudaError_t launch_fill_dense(int nQ, int nAtom, const float* coors, const float* mincoors,
                              const AtomParam* params, int nVdwUsed, int X, int Y, int Z,
                              float spacing, float* out, cudaStream_t s);
cudaError_t launch_conj_mult(const float2* pot, float2* lig, int odist, int K, int Q,
                             cudaStream_t s);
cudaError_t launch_sum_grids(const float2* lig, float2* sum, int K, int odist, int idist,
                             int Q, cudaStream_t s);
// FP64 direct re-score of poses.
cudaError_t launch_rescore_fp64(int n, int K, float spacing, const float* grids,
                                const float* coords, const AtomParam* params,
                                const ConfDesc* confs, const RotDesc* rots, const int* tidx,
                                int npose, double* energy, cudaStream_t s);

// Precision form: x pass as a split-BF16 circulant contraction on the tensor cores.
cudaError_t launch_ptilde(int n, int K, const float2* yz, float2* pt, cudaStream_t s);
cudaError_t launch_xpass_tc(const WaveArgs& a, const float2* pt, cudaStream_t s);
size_t xpass_tc_smem_bytes(int n, int K, int Lb);
// tcgen05 variant of the precision x pass (n = 64)
bool umma_supported(int n, int Lb);
cudaError_t launch_xpass_umma(const WaveArgs& a, const float2* pt, cudaStream_t s);
// tcgen05 x pass with streamed operands (n = 64): the operator image is built once per receptor
// from P~, the ligand rows come from the plane kernel (WaveArgs.lop)
bool stream_supported(int n, int Lb);
size_t stream_top_bytes(int n, int K);
size_t stream_lop_bytes_per_rotation(int n, int K, bool f16);
// plane group of the B layout the shared-memory streamed x pass writes (CDK_B_GROUP overrides)
int stream_bgroup();
// f16_scale: nullptr = the split-BF16 image; else the split-FP16 image of P~ * f16_scale[k]
cudaError_t launch_top_build(int n, int K, const float2* pt, void* top, const float* f16_scale,
                             cudaStream_t s);
cudaError_t launch_xpass_stream(const WaveArgs& a, const void* top, cudaStream_t s);
// true when launch_spread_yz takes the direct plane path (the only one that can write lop)
bool direct_planes(const WaveArgs& a);

// tcgen05 x pass with the Hankel operator resident in shared memory (any n, ligand box <= 32
// planes): its shape for (n, K, box, form) and its launch (k_tile_plan, then the x pass)
struct HankelPlan {
  int cols;         // spectral columns per CTA (1 or 2)
  int G;            // 128-byte groups of one Hankel buffer
  int jc;           // 8-plane K-steps of the ligand box
  int nb;           // ring stages
  int ks;           // K-steps per ring stage (1 to 4)
  size_t smem;      // dynamic shared memory per CTA
  int ctas_per_sm;  // 1 or 2
};
// nb_cap > 0: at most that many ring stages (the autotuner's candidates); ks_pref > 0: that many
// K-steps per stage
bool hankel_plan(int n, int K, int Lb, bool f16, int cols_pref, HankelPlan* out, int nb_cap = 0,
                 int ks_pref = 0);
cudaError_t launch_xpass_hankel(const WaveArgs& a, const float2* pt, const float* f16_scale,
                                const HankelPlan& p, cudaStream_t s);
// the B layout the plan's x pass writes (and the inverse (y,z) kernels then read): one column per
// CTA writes single-column groups of 4 planes, two columns column-pair groups
void hankel_b_layout(const HankelPlan& p, WaveArgs& a);
// the stage plan of every 128-rotation tile of a wave into the tile's first RotRec
cudaError_t launch_tile_plan(const WaveArgs& a, int jc, cudaStream_t s);

// Digit-reversed position of natural frequency k for the radix plan of length n.
int fft_position(int n, int k);

// Number of kernel launches one wave issues.
constexpr int kLaunchesPerWave = 5;

void set_error(const std::string& msg);

// Read-only view of a context's resident state, for entry points that live outside capi.cu.
struct CtxView {
  int dev, n, K;
  float spacing;
  int col_tile_opt, max_atoms;
  const float2* phat;
  const float2* tw;
  const int* kyof;
  unsigned int* h_misc;  // pinned host scratch of the context (8 words)
  cudaStream_t stream;
  int form;              // CDK_FORM_*
  int tc_variant;        // opts.reserved[3]
  int hx_shape;          // opts.reserved[5]
  const void* top;       // operator image of the streamed tensor-core x pass (or null)
  const float2* ptilde;  // precision forms: P~ [ncol][K][n], the Hankel x pass's operator source
  const float* grids;    // receptor grids [K][n][n][n] (FP64 re-scores)
  bool tiebreak;         // precision forms: FP64 near-tie break of the argmin
  float lscale[KMAX];    // split-FP16 form: ligand scale 2^sigma_k per channel
};

}  // namespace cdk

struct cdk_ctx;
namespace cdk {
// Fills *v from the context; returns false for a null context.
bool ctx_view(const cdk_ctx* c, CtxView* v);
// Builds the context's operator image for the streamed tensor-core x pass if it does not exist
// yet (precision-form contexts at n = 64); synchronises the context stream. CDK_* status.
int ctx_ensure_top(cdk_ctx* c);
}  // namespace cdk
