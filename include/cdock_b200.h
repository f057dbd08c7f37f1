/* cdock_b200.h -- C-ABI of the B200 FFT translational-rotational search.
 *
 * The reference (CDOCKER) has no library boundary for this path: the search runs inline in
 * each driver's main() (src/TranRotaConfSearchNoMini.cu:156-464, and the same block in
 * src/TranRotaSearch.cu:111-350), and its only declared GPU interface is include/kernel.h
 * (ConjMult, SumGrids). The entry points below are that path cut at its natural seams, with
 * plain pointers and sizes; each comment names the reference code it replaces.
 *
 * Conventions
 *  - Every function returns an int status (CDK_OK = 0) and never exits the process;
 *    cdk_last_error() returns the message of the last failure on the calling thread.
 *  - Grids are float [K][nx][ny][nz], z fastest, the reference's usedGridValues layout
 *    (src/TranRotaConfSearchNoMini.cu:135-146): K-1 vdW grids, then the electrostatic grid.
 *  - Atom slots are the position of each atom's vdW grid among the K-1 used vdW grids, as
 *    produced by GetIdxOfAtomsForVdwRadius (src/GetIdxOfAtomsForVdwRadius.cpp:4-35).
 *  - A context owns all device memory it uses. Contexts are independent; one context must not
 *    be driven from two host threads at once.
 *  - stream arguments are cudaStream_t passed as void* (NULL = the context's own stream).
 */
#ifndef CDOCK_B200_H
#define CDOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CDK_OK 0
#define CDK_ERR_INVALID 1     /* bad argument */
#define CDK_ERR_CUDA 2        /* a CUDA call failed */
#define CDK_ERR_NOMEM 3       /* device allocation failed */
#define CDK_ERR_UNSUPPORTED 4 /* grid size / K outside what the kernels are built for */
#define CDK_ERR_OVERFLOW 5    /* a rotation's ligand box exceeded the planned box */
#define CDK_ERR_IO 6          /* file could not be read or parsed */
#define CDK_ERR_BUSY 7        /* serving queue full / admission refused */

#define CDK_FORM_FP32 0   /* FP32 radix FFT passes (the plain form) */
#define CDK_FORM_BF16X3 1 /* split-BF16 (hi*hi + hi*lo + lo*hi) DFT contractions, FP32 acc. */
#define CDK_FORM_FP16X2 2 /* split-FP16 operator x FP16 ligand rows (two products), per-channel
                             power-of-two scaling, FP32 acc.: about 1e-4 relative error; half the
                             ligand bytes and two thirds of the MMAs of BF16X3. Ligands of at most
                             96 atoms with a box of at most 32 planes; a search outside that
                             returns CDK_ERR_UNSUPPORTED (BF16X3 covers every ligand) */

typedef struct cdk_ctx cdk_ctx;

typedef struct cdk_opts {
  int device;          /* CUDA device ordinal */
  int form;            /* CDK_FORM_* */
  int wave_rotations;  /* rotations per launch wave; 0 = pick automatically */
  int max_atoms;       /* largest ligand (atoms) this context will see; 0 = 256 */
  int col_tile;        /* spectral columns per CTA in the x pass; 0 = autotuned default */
  int use_graphs;      /* 1 = replay each wave through a captured CUDA graph */
  int reserved[8];     /* [0] = 1: time every kernel with events (cdk_ctx_stats [8..12]);
                          [1] bit 0: spread planes through the radix FFT instead of the direct
                          separable evaluation; bit 1: the inverse (y,z) kernel with
                          block-wide radix stages at every n; bit 2: the one with warp-local
                          line transforms at every n (default: block stages at n <= 64,
                          warp-local lines at n >= 96); [2] = 1: autotune the x pass on the first wave
                          of each new ligand box; [3] precision-form x pass: 0 = automatic
                          (ligands <= 96 atoms, box <= 32 planes: tcgen05 with the Hankel
                          operator resident in shared memory; else the next one); 1 = mma.sync;
                          2 = tcgen05 with operands built inside the kernel (n = 64);
                          3 = streamed operator tiles (n = 64); 4 = the Hankel kernel;
                          [4] = 1: keep the rotations in the given order in the streamed
                          tensor-core x pass (by default they are grouped by the ligand-box
                          chunks their channels reach, which changes no result);
                          [5] Hankel x pass shape: bits 0-1 columns per CTA (0 = automatic,
                          1, or 2 at n <= 64), bits 2-4 K-steps per ring stage (0 = automatic,
                          1 to 4), bit 5: ligand rows copied per rotation by the producer
                          threads, bit 6 (the default where the driver provides the
                          tensor-map encoder): ligand rows written by the plane kernel in
                          128-rotation row sets that the x pass loads by tensor copies (the
                          same results either way);
                          [6] precision forms: poses per wave re-scored in FP64
                          (cdk_ctx_top_poses): 0 = 8 (none in the FP32 form), -1 = none,
                          1..32; [7] = 1: no FP64 near-tie break of the argmin in the
                          precision forms (by default, when a rotation's two best translations
                          lie within 1e-3 (split-FP16) or 1e-4 (split-BF16) x max(|E|, 1) of
                          each other, both are re-scored in FP64 and the lower is kept) */
} cdk_opts;

/* Library version string. */
const char* cdk_version(void);

/* Message of the last failure on this thread (empty if none). Returns the message length. */
int cdk_last_error(char* buf, size_t cap);

/* Fills *opts with defaults. */
void cdk_opts_default(cdk_opts* opts);

/* Upload the K receptor grids and transform them once; the K spectra stay resident.
 * Replaces src/TranRotaConfSearchNoMini.cu:156-199 (cufftPlanMany R2C + H2D + ExecR2C).
 * nx == ny == nz in {32, 64, 96, 128}; 2 <= K <= 16. grids: host pointer. */
int cdk_ctx_create(int nx, int ny, int nz, float spacing, int K, const float* grids,
                   const cdk_opts* opts, cdk_ctx** out);
int cdk_ctx_destroy(cdk_ctx* ctx);

/* Whole search over nConf conformers x nQ rotations, host buffers in and out.
 * Replaces src/TranRotaConfSearchNoMini.cu:352-464 (rotate, bounding box, FillLigandGrid,
 * H2D, R2C, ConjMult, SumGrids, C2R, D2H, host min/argmin). Rotation i of conformer c is
 * quats[(c*nQ + i)*4 .. +4]; results minE[c*nQ+i] and idx[(c*nQ+i)*3 .. +3] follow the
 * reference: minimum over the window [0, n - int(len/h) - 2) per axis of the correlation
 * energy, first minimum in x-major order; +inf and -1 for an empty window.
 * coor: [nConf][nAtom][3]; charge, eps: [nAtom]; slot: [nAtom] in 0..K-2. */
int cdk_search(cdk_ctx* ctx, int nAtom, int nConf, const float* coor, const float* charge,
               const float* eps, const int* slot, int nQ, const float* quats, float* minE,
               int* idx, void* stream);

/* Same search with every buffer already in device memory (d_ prefix = device pointer);
 * no host<->device copies and no synchronisation beyond stream order. */
int cdk_search_device(cdk_ctx* ctx, int nAtom, int nConf, const float* d_coor,
                      const float* d_charge, const float* d_eps, const int* d_slot, int nQ,
                      const float* d_quats, float* d_minE, int* d_idx, void* stream);

/* cdk_search_device without any device allocation. It has no counterpart in the reference.
 * For callers that cannot let the library call cudaMalloc when they search (real-time loops
 * that must not hit the allocator's device-wide synchronisation, device memory owned by a
 * pool that forbids outside allocations): the wave and table scratch that cdk_search_device
 * grows with cudaMalloc comes instead from one file-scope device array of
 * CDK_NOALLOC_SCRATCH_BYTES (64 MiB), held by every GPU that loads the library until exit.
 * FP32-form contexts only: a context of another form returns CDK_ERR_UNSUPPORTED. Rotations
 * run in waves that fit the array; a search whose single rotation does not fit returns
 * CDK_ERR_UNSUPPORTED. The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it; the cache does not survive cudaDeviceReset. The call
 * synchronises its stream twice (ligand-box plan, overflow count). Calls share the array:
 * calls that overlap on the GPU race; serialise them. Otherwise the same arguments, results
 * and errors as cdk_search_device on an FP32 context. */
#define CDK_NOALLOC_SCRATCH_BYTES (64u << 20)
int cdk_search_device_noalloc(cdk_ctx* ctx, int nAtom, int nConf, const float* d_coor,
                              const float* d_charge, const float* d_eps, const int* d_slot,
                              int nQ, const float* d_quats, float* d_minE, int* d_idx,
                              void* stream);

/* FP64 direct re-score of given poses (rotation + translation index) against the resident
 * receptor grids: E = sum_k sum_atoms sum_corners w * P_k(g + t), accumulated in double.
 * Host buffers. rot_conf[i] picks the conformer, quats[i*4..], tidx[i*3..] the translation. */
int cdk_rescore_fp64(cdk_ctx* ctx, int nAtom, int nConf, const float* coor,
                     const float* charge, const float* eps, const int* slot, int nPose,
                     const int* rot_conf, const float* quats, const int* tidx, double* energy,
                     void* stream);

/* Dense ligand-grid fill on the GPU with FillLigandGrid's semantics
 * (src/FillLigandGrid.cpp:7-120): rotated coords [nQ][nAtom][3] and their min corners
 * [nQ][3] in, out[nQ][nVdwUsed+1][x][y][z] (host, overwritten; the reference wants it
 * pre-zeroed, this call zeroes it). */
int cdk_fill_ligand_grid(int nQ, int nAtom, const float* coors, const float* mincoors,
                         const float* charge, const float* eps, const int* slot, int nVdwUsed,
                         int x, int y, int z, float spacing, float* out);

/* kernel.h-compatible spectral kernels on device pointers (include/kernel.h:9-11), with
 * bounds checks. d_potential_F: [K][odist] complex; d_ligand_F: [Q][K][odist] complex.
 * cdk_conj_mult: d_ligand_F[q,k,f] <- conj(d_ligand_F[q,k,f]) * d_potential_F[k,f]
 *   (src/kernel.cu:5-14).
 * cdk_sum_grids: d_sum_F[q,f] = sum_k d_ligand_F[q,k,f] / sqrtf(idist) (src/kernel.cu:16-30). */
int cdk_conj_mult(const void* d_potential_F, void* d_ligand_F, int odist, int K, int Q,
                  void* stream);
int cdk_sum_grids(const void* d_ligand_F, void* d_sum_F, int K, int odist, int idist, int Q,
                  void* stream);

/* Host helpers with the reference's semantics (bit-exact). */

/* nConf x nQ Shoemake quaternions from one std::mt19937_64 seeded with `seed`, drawn in turn
 * (src/QuaternionUniformSampling.cpp:5-24; the driver's shared generator, :203-204, :323). */
int cdk_quaternion_uniform_sampling(uint64_t seed, int nConf, int nQ, float* out);

/* FilterQuaternions (src/FilterQuaternions.cpp:11-83): keeps rotations whose rotated box is
 * shorter than the grid lengths; if more than maxN pass, std::random_shuffle (driven by the
 * process-wide rand()) and keep the first maxN. out: nQ*4 capacity; returns the count via
 * *count. */
int cdk_filter_quaternions(const float* coor, int nAtom, int nQ, const float* quats,
                           float gridLenX, float gridLenY, float gridLenZ, int maxN,
                           float* out, int* count);

/* GetIdxOfAtomsForVdwRadius (src/GetIdxOfAtomsForVdwRadius.cpp:4-35) + the driver's grid
 * compaction (src/TranRotaConfSearchNoMini.cu:126-146): per-atom slot among the used vdW
 * grids, the used grid indices (ascending), and their count via *nUsed. */
int cdk_vdw_slots(int nAtom, const float* radii, int nVdw, const float* gridRadii,
                  int* usedIdx, int* atomSlot, int* nUsed);

/* sort_index (include/GeneDiverseConformations.h:9-20, used on the per-rotation minima at
 * src/TranRotaConfSearchNoMini.cu:469): out[0..n) = indices of v in ascending order by
 * std::sort with strict <, so equal values come out in the same (unstable) order as the
 * reference's call. */
int cdk_sort_index(const float* v, long n, long* out);

/* Pose of one rotation at its best translation (src/TranRotaConfSearchNoMini.cu:473-487):
 * out[a] = Rotate(quat, coor[a]) + gridMin - mincoor + idx * spacing, in double.
 * gridMin = mid - len/2 of the grid file (:149-151). */
int cdk_pose_coordinates(int nAtom, const float* coor, const float* quat, const double* gridMin,
                         float spacing, const int* idx, double* out);

/* Diverse-conformer selection: the greedy leader clustering of GeneDiverseConformations
 * (src/GeneDiverseConformations.cpp:84-111), on the GPU. Conformers coor[nConf][nAtom][3]
 * (double, Angstrom, as OBMol coordinates) are taken in energy order (sort_index<double>,
 * include/GeneDiverseConformations.h:9-20); the lowest is the first centre; each following one
 * is a new centre when its superposition RMSD to every centre so far is > cutoff (the reference
 * uses 1.5). The loop stops when the centre count equals maxCenters, tested after each
 * candidate from the second on, as the reference does. RMSD: minimum over rotations after
 * centring, over the atoms with atomMask[a] != 0 (NULL = all atoms), without symmetry
 * permutations (OBAlign, absent here, also tries automorphisms of symmetric molecules).
 * centers: capacity nConf; receives conformer indices in selection order, *nCenters their
 * count. nConf <= 32768. Uses the current CUDA device. */
int cdk_cluster_conformers(int nConf, int nAtom, const double* coor, const double* energy,
                           const unsigned char* atomMask, double cutoff, int maxCenters,
                           int* centers, int* nCenters);

/* The RMSD the clustering compares, for all pairs: out[i*nConf + j] = min RMSD of conformer i
 * (reference) and j (target) after superposition. nConf <= 16384. */
int cdk_pair_rmsd(int nConf, int nAtom, const double* coor, const unsigned char* atomMask,
                  double* out);

/* ReadGrids (src/ReadGrids.cpp:6-68): header ints [numGrids, x, y, z], floats
 * [midx, midy, midz, xlen, ylen, zlen, spacing, restraint_k]; radii (numGrids-1) and values
 * (numGrids*x*y*z) are written when the capacities suffice. Pass NULL buffers to size first. */
int cdk_read_grids(const char* path, int* hdr_i, float* hdr_f, float* radii, long radii_cap,
                   float* values, long values_cap);

/* Writes grids in the same text format (3 title lines, header, radii, per grid a header line
 * and x y z value lines, z fastest). */
int cdk_write_grids(const char* path, int numGrids, int x, int y, int z, const float* mid,
                    const float* len, float spacing, float restraint_k, const float* radii,
                    const float* values);

/* Seeded synthetic receptor potential grids: nVdw soft-core capped LJ grids at the given probe
 * radii and one distance-dependent-dielectric Coulomb grid (eps(r) = 4r, capped at +-elecCap),
 * from receptor atoms xyz[nAtom][3], radius, sqrt-epsilon and charge. Grid point (i,j,k) is
 * origin + (i,j,k)*spacing. out: [nVdw+1][n][n][n]. Host, multithreaded. */
int cdk_synth_receptor_grids(int n, float spacing, const float* origin, int nAtom,
                             const float* xyz, const float* radius, const float* sqrtEps,
                             const float* charge, int nVdw, const float* probeRadii,
                             float vdwCap, float elecCap, float cutoff, float* out);

/* The same grids computed on CUDA device `device` (one thread per grid point, double
 * accumulation with round-to-nearest operations in the host function's order, so the output
 * is bit-identical to cdk_synth_receptor_grids). Host inputs and output; nVdw <= 15. The
 * reference reads these grids from CHARMM-written files (src/ReadGrids.cpp:6-68); this
 * replaces the CHARMM grid-generation step upstream of cdk_read_grids. */
int cdk_receptor_grids_gpu(int device, int n, float spacing, const float* origin, int nAtom,
                           const float* xyz, const float* radius, const float* sqrtEps,
                           const float* charge, int nVdw, const float* probeRadii,
                           float vdwCap, float elecCap, float cutoff, float* out);

/* ---- serving: continuous batching over one resident receptor ----
 * A server owns a worker thread and a stream on the context's device. Requests (a ligand
 * with its conformers and rotations) are admitted when their inputs and outputs fit the
 * server's device arena, in FIFO order; the worker packs the rotations of all admitted
 * requests into shared waves, so requests that arrive while others run join the next wave.
 * Results are the same as cdk_search on the request alone. The context must outlive the
 * server. The reference has no serving layer (it searches one ligand per process run). */
typedef struct cdk_server cdk_server;
typedef struct cdk_server_opts {
  size_t arena_bytes;  /* device memory for request inputs/outputs (admission budget) */
  int wave_rotations;  /* rotations per shared wave */
  int max_box;         /* largest ligand box edge (grid cells) a request may need */
  int max_atoms;       /* largest ligand */
  int max_conformers;  /* conformer slots across admitted requests */
  int max_waiting;     /* queued (not yet admitted) requests before submit returns BUSY */
  int reserved[4];     /* [0] = w > 0: test switch, the host sets the device-wait fault word of
                          wave number w-1 after its kernels (every request in it then fails
                          with CDK_ERR_CUDA); 0 in production */
} cdk_server_opts;
void cdk_server_opts_default(cdk_server_opts* opts);
int cdk_server_create(cdk_ctx* ctx, const cdk_server_opts* opts, cdk_server** out);
/* Copies the request; returns a ticket. CDK_ERR_BUSY when the wait queue is full. */
int cdk_server_submit(cdk_server* s, int nAtom, int nConf, const float* coor,
                      const float* charge, const float* eps, const int* slot, int nQ,
                      const float* quats, uint64_t* ticket);
/* Waits up to wait_ms (-1: forever, 0: no wait). CDK_OK: results copied (minE[nConf*nQ],
 * idx[nConf*nQ][3]) and timing[0..2] = queue, run, total ms; the ticket is then released.
 * CDK_ERR_BUSY: still running. A finished request that failed returns its own status (results
 * are still copied and the ticket released): CDK_ERR_OVERFLOW when a rotation of it left the
 * planned ligand box, CDK_ERR_UNSUPPORTED when a scaled ligand value of it left the FP16 range
 * of the split-FP16 form (those rotations read minE = NaN and idx = -2 or -3), CDK_ERR_CUDA when
 * a wave that held its rotations failed to launch or a bounded device wait in it gave up.
 * Errors are attributed per request: other requests of the same wave are unaffected by a
 * per-rotation cause. */
int cdk_server_poll(cdk_server* s, uint64_t ticket, int wait_ms, float* minE, int* idx,
                    double* timing);
/* [0] waves, [1] rotations, [2] kernel launches, [3] completed requests, [4] p50 latency ms,
 * [5] p99 latency ms, [6] waiting requests, [7] admitted requests in flight, [8] waves run on
 * the tensor-core x pass (precision-form contexts: waves whose ligand box is <= 32 planes and
 * whose ligands have <= 96 atoms, at any grid size; the others run the FP32 x pass). */
int cdk_server_stats(cdk_server* s, double* out, int n);
int cdk_server_destroy(cdk_server* s);

/* Counters of the last search on this context (n <= CDK_NSTATS values):
 * [0] kernel launches, [1] waves, [2] rotations, [3] device ms of the search (events on the
 * search stream), [4] planned ligand box edge, [5] rotations per wave, [6] (y,z) planes the
 * spread kernel transformed, [7] window planes the x pass wrote, [8..12] device ms per kernel
 * kind (prep, spread_yz, xpass, yz_inv_argmin, finalize) when the context was created with
 * opts.reserved[0] = 1 (events around every launch), else 0; [13] x-pass column tile,
 * [14] x-pass rotations per CTA, [15] graph state (0 off, 1 shape seen, 2 replaying),
 * [16] x-pass kind (0 FP32 radix, 1 mma.sync, 2 tcgen05 with in-kernel operand builds,
 * 3 tcgen05 with streamed operator tiles (64^3), 5 the same in the split-FP16 form,
 * 6 tcgen05 with the resident Hankel operator, 7 the same in the split-FP16 form),
 * [17] tensor-core K-steps the x pass issued per spectral column (one step = the MMAs of one
 * 8-plane chunk of one channel for one column and 128 rotations), [18] Hankel x pass: issued
 * MMA work in units of 128 x 8 x 16 multiply-adds (32,768 flops), [19] rotations whose two
 * best translations lay within the near-tie tolerance and were re-scored in FP64, [20] of them,
 * those whose translation the FP64 re-score changed. */
#define CDK_NSTATS 21
int cdk_ctx_stats(cdk_ctx* ctx, double* out, int n);

/* The precision forms' FP64 re-score of each wave's lowest poses (the north star's top-k per
 * rotation batch; opts.reserved[6] sets k): for the last search, *count = waves x k entries, wave
 * by wave, each ascending in energy: rot[i] the rotation (c*nQ + q), minE[i] the search's
 * energy, idx[i*3..] its translation, e64[i] the FP64 direct grid-energy sum of that pose
 * (rot = -1 for slots of a wave with fewer valid rotations). Up to cap entries are copied. */
int cdk_ctx_top_poses(cdk_ctx* ctx, int cap, int* rot, float* minE, int* idx, double* e64,
                      int* count);

#ifdef __cplusplus
}
#endif
#endif /* CDOCK_B200_H */
