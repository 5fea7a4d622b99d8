/*
 * argot_b200.h -- C ABI of libargot_b200.so, a B200 (sm_100a) implementation
 * of ARGOT's point-source radiative-transfer hot path:
 *
 *   calc_optical_depth   per-segment mesh march -> HI/HeI/HeII columns
 *   accum_optical_depth  stitching of segment columns into light rays
 *   calc_photoion_rate   256-bin photo-ionisation / heating integral per cell
 *
 * Two layers are exported.
 *
 * 1. Drop-in entry points with the reference's exact names and signatures
 *    (ARGOT src/prototype.h).  The reference's structs are only
 *    forward-declared here, so a C host that includes ARGOT's own headers can
 *    include this file too.  ARGOT fixes its struct layouts and its rate
 *    formula with preprocessor flags (src/Makefile:149-196), so the library
 *    is built once per flag set, against byte-identical mirrors of the
 *    structs for that set (NGRID_NU=256, NSEG_PER_RAY=5, NMAX_CUDA_DEV=4):
 *      libargot_b200.so          -D__HELIUM__ -D__PHOTON_CONSERVING__ (the
 *                                default; also carries the device API of 2.)
 *      libargot_b200_h2_pc.so    -D__HYDROGEN_MOL__ -D__PHOTON_CONSERVING__
 *                                (the set ARGOT's own Makefile compiles)
 *      libargot_b200_he_h2_pc.so, libargot_b200_he.so (no photon
 *      conservation), libargot_b200_he_pc_cosmo.so (-D__COSMOLOGICAL__), ...
 *    (argot_b200/build.py builds any other combination on request).  A host
 *    links the one its own flags select; argot_b200_flagset() names it and
 *    argot_b200_abi_check() verifies the caller's struct sizes at run time.
 *    Mesh dimensions are read from run_param at run time, so one library
 *    serves every NMESH_* build.  These entry points use GPU 0 of the
 *    caller's cuda_param (one rank, one GPU).
 *
 * 2. A device-resident API (argot_b200_*): plain pointers, sizes and a CUDA
 *    stream; caller-owned device buffers; no reference structs.  This is the
 *    B200 fast path (rays held as 4-byte words, target-blocked, emitter
 *    spectra by index), used by the benchmark and callable from any host
 *    language through the C ABI.
 *
 * Every argot_b200_* function returns 0 on success or a negative
 * ARGOT_B200_E* code; the drop-in void functions record their status, which
 * argot_b200_last_error() returns.  No function traps the device.
 */
#ifndef ARGOT_B200_H
#define ARGOT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ARGOT_B200_API __attribute__((visibility("default")))
#else
#define ARGOT_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define ARGOT_B200_OK 0
#define ARGOT_B200_EINVAL (-1)      /* bad argument / size / layout         */
#define ARGOT_B200_ECUDA (-2)       /* a CUDA runtime call failed           */
#define ARGOT_B200_ENOMEM (-3)      /* device or pinned allocation failed   */
#define ARGOT_B200_EDEVICE (-4)     /* a kernel reported an internal error  */
#define ARGOT_B200_ENOTSUP (-5)     /* option not supported                 */

/* status of the last call made by this host thread */
ARGOT_B200_API int argot_b200_last_error(void);
ARGOT_B200_API const char *argot_b200_error_string(int code);

/* library / ABI identification */
ARGOT_B200_API const char *argot_b200_version(void);
/* the flag set this build's drop-in follows, e.g. "helium, photon
 * conserving" or "h2, photon conserving" */
ARGOT_B200_API const char *argot_b200_flagset(void);
/* sizes[10]: ray_segment, light_ray, light_ray_IO, radiation_src,
 * fluid_mesh, prim_chem, run_param, cross_section, freq_param,
 * photoion_rate as the library was compiled */
ARGOT_B200_API void argot_b200_struct_sizes(uint64_t *sizes);
/* returns 0 when the caller's sizeof() values (same order) match */
ARGOT_B200_API int argot_b200_abi_check(const uint64_t *caller_sizes, int n);

/* ============================================================ 1. drop-in */
struct ray_segment;
struct light_ray;
struct light_ray_IO;
struct fluid_mesh;
struct run_param;
struct cuda_mem_space;
struct cuda_param;
struct omp_param;
struct mpi_param;

/* Replaces src/calc_optical_depth_cuda.cu:29-144 (declared at
 * src/prototype.h:124).  Overwrites seg[0..run->nseg).optical_depth_* (every
 * column of the build's flag set: HI, HeI, HeII, HM, H2I, H2II as present)
 * in host memory before returning.  Reads the mesh from
 * cuda_mem[0].mesh_dev (device AoS struct fluid_mesh, filled by the caller's
 * send_mesh_data) and the domain geometry from *this_run (host copy). */
ARGOT_B200_API void calc_optical_depth_cuda(struct ray_segment *seg, struct cuda_mem_space *cuda_mem,
                             struct cuda_param *this_cuda, struct run_param *this_run);

/* Replaces src/calc_photoion_rate_cuda.cu:92-216 (src/prototype.h:125).
 * Fills ray_IO from ray as the reference does, and ADDS each ray's rates to
 * cuda_mem[0].mesh_dev[target].prev_chem: every Gamma and Heat field of the
 * build's flag set, by the photon-conserving or the plain formula and with
 * the scale-factor terms as the flags select (calc_photoion_rate.c:93-439,
 * the H2 Lyman-Werner term included), in FP64.  The frequency grid and the
 * cross sections are the caller's (this_run->freq, this_run->csect). */
ARGOT_B200_API void calc_photoion_rate_cuda(struct cuda_mem_space *cuda_mem, struct light_ray *ray,
                             struct light_ray_IO *ray_IO, struct cuda_param *this_cuda,
                             struct run_param *this_run);

/* Replaces src/calc_photoion_rate_cuda.cu:45-62 (src/prototype.h:93):
 * zeroes every rate field of prev_chem in cuda_mem[0].mesh_dev. */
ARGOT_B200_API void zero_out_photoion_rate_cuda(struct cuda_mem_space *cuda_mem,
                                 struct cuda_param *this_cuda, struct run_param *this_run);

/* Replaces src/accum_optical_depth.c:14-167 (src/prototype.h:47) for a
 * single-rank run: every segment's columns go to ray[seg.ray_indx], rays
 * without a segment get zero.  A host routine (the columns are already in
 * host memory after calc_optical_depth_cuda).  An executable that still
 * links the reference's accum_optical_depth.o keeps using its own: the
 * executable's definition takes precedence over the shared library's. */
ARGOT_B200_API void accum_optical_depth(struct light_ray *ray, struct ray_segment *seg,
                         struct run_param *this_run, struct omp_param *this_omp);

/* Arithmetic mode of the drop-in march: ARGOT_B200_MARCH_REFERENCE (default)
 * reproduces the reference's FP32 operation order bit for bit;
 * ARGOT_B200_MARCH_KAHAN uses the parametric FP32 march with compensated
 * column sums (closer to an FP64 evaluation). */
#define ARGOT_B200_MARCH_REFERENCE 0
#define ARGOT_B200_MARCH_KAHAN 1
ARGOT_B200_API int argot_b200_set_dropin_march_mode(int mode);

/* Replaces src/smooth_photoion_rate.c:27-1588 as built with __USE_GPU__
 * (src/prototype.h:89) on a single rank.  Smooths every rate field of
 * cuda_mem[0].mesh_dev[].prev_chem in place on the
 * device, bit-identical to the reference's host smoothing (27 cells, centre
 * weighted by 30, times 1/56), so the rates stay in HBM for the GPU
 * chemistry (src/chemistry.cu) that reads mesh_dev next; then, when mesh is
 * not NULL, writes the smoothed values into mesh[].prev_chem as the
 * reference does.  this_mpi is not used (no neighbour ranks).  The mesh
 * faces follow argot_b200_set_dropin_smooth_faces. */
ARGOT_B200_API void smooth_photoion_rate(struct fluid_mesh *mesh, struct run_param *this_run,
                                         struct cuda_mem_space *cuda_mem, struct cuda_param *this_cuda,
                                         struct mpi_param *this_mpi);

/* Faces of the drop-in smoothing: ARGOT_B200_FACES_ISOLATED (default; ARGOT
 * built with -D__ISOLATED__, its Makefile's default: a face cell stands in
 * for its missing neighbour) or ARGOT_B200_FACES_PERIODIC (the periodic
 * image). */
#define ARGOT_B200_FACES_PERIODIC 0
#define ARGOT_B200_FACES_ISOLATED 1
ARGOT_B200_API int argot_b200_set_dropin_smooth_faces(int faces);

/* ================================================= 2. device-resident API */

/* Domain geometry of one rank, in the reference's terms (run_param). */
typedef struct argot_b200_grid {
  int nx, ny, nz;                  /* local cells per axis                  */
  int ix0, iy0, iz0;               /* global index of local cell (0,0,0)    */
  float xmin, ymin, zmin;          /* global box lower corner               */
  float xmax, ymax, zmax;          /* global box upper corner               */
  float xmin_local, ymin_local, zmin_local;
  float dx, dy, dz;                /* cell size                             */
  double lunit;                    /* length unit [cm]                      */
  double denstonh;                 /* code density -> n_H [cm^-3]           */
} argot_b200_grid;

/* Packed cell fields (32 bytes per cell, 16-byte aligned): first ncell
 * float4 {n_HI, n_HeI, n_HeII, 0} in code density units, the products
 * rounded exactly as the reference forms them per crossing
 * (calc_optical_depth.c:150-155) -- the march reads only these; then ncell
 * float4 {dens, fHI, fHeI, fHeII}, read by the rate stage at the target
 * cell.  Cell index iz + nz*(iy + ny*ix). */

/* from separate device arrays (dens, fHI, fHeI, fHeII: ncell floats each) */
ARGOT_B200_API int argot_b200_pack_fields(const argot_b200_grid *g, const float *dens, const float *fHI,
                           const float *fHeI, const float *fHeII, void *packed_dev,
                           void *stream);
/* from a device array of the reference's struct fluid_mesh (156 B/cell);
 * ARGOT_B200_ENOTSUP in a build for a flag set without helium or with H2 or
 * the scale factor (the device path carries HI, HeI and HeII only) */
ARGOT_B200_API int argot_b200_pack_fluid_mesh(const argot_b200_grid *g, const void *mesh_dev,
                               void *packed_dev, void *stream);

/* ---- emitters (tree nodes and sources) and the oct-tree ---------------- */

/* Host-side oct-tree over the sources, built as the reference's
 * construct_tree (setup_light_ray_tree.c:465-571): Morton keys of 21 bits
 * per axis, luminosity-weighted centres, summed spectra.  The tree is then
 * uploaded and walked on the device. */
typedef struct argot_b200_tree argot_b200_tree;

/* src_pos: nsrc x 3 floats; spectra: nsrc x 256 photon rates [s^-1 per bin]
 * (setup_photon_rate output); theta: opening angle. */
ARGOT_B200_API int argot_b200_tree_build(const argot_b200_grid *g, int nsrc, const float *src_pos,
                          const double *spectra, float theta, argot_b200_tree **out);
ARGOT_B200_API void argot_b200_tree_free(argot_b200_tree *t);
/* number of emitters = tree nodes + sources; nodes come first */
ARGOT_B200_API int argot_b200_tree_num_emitters(const argot_b200_tree *t);
ARGOT_B200_API int argot_b200_tree_num_nodes(const argot_b200_tree *t);
/* emitter table for the kernels, host side:
 *   pos4:     n_emit x 4 floats (x, y, z, 0)
 *   spec64:   n_emit x 256 doubles (photon rate per bin)
 * either pointer may be NULL */
ARGOT_B200_API int argot_b200_tree_emitters(const argot_b200_tree *t, float *pos4, double *spec64);

/* Device copy of the walkable tree (nodes, leaf source lists) and of the
 * emitter table; must be freed with argot_b200_dev_tree_free. */
typedef struct argot_b200_dev_tree argot_b200_dev_tree;
ARGOT_B200_API int argot_b200_dev_tree_upload(const argot_b200_tree *t, argot_b200_dev_tree **out,
                               void *stream);
ARGOT_B200_API void argot_b200_dev_tree_free(argot_b200_dev_tree *d);
/* The same device tree built on the device from the sources' positions
 * (nsrc x 3 floats) and spectra (nsrc x 256 doubles) in device memory:
 * Morton keys, a stable radix sort, node enumeration in depth-first
 * preorder, node sums level by level from the leaves up.  Bit-identical
 * to argot_b200_tree_build + argot_b200_dev_tree_upload (the reference's
 * construct_tree, setup_light_ray_tree.c:465-571); the surrogate's
 * per-emitter inputs (argot_b200_dev_tree_set_blackbody) still need the
 * host tree.  Allocates scratch and the tree; synchronises `stream`. */
ARGOT_B200_API int argot_b200_dev_tree_build(const argot_b200_grid *g, int nsrc, const float *src_pos_dev,
                                             const double *spectra_dev, float theta, argot_b200_dev_tree **out,
                                             void *stream);
/* node and emitter counts and the emitters' bounding box (lo xyz, hi xyz) */
ARGOT_B200_API int argot_b200_dev_tree_info(const argot_b200_dev_tree *d, int *n_nodes, int *n_emit,
                                            float *bounds6);
/* host copies of a device tree's arrays (any pointer may be NULL): emitter
 * positions (n_emit x 4 floats), FP64 spectra (n_emit x 256), the nodes
 * (n_nodes x 8 words: centre x y z, side as floats; sources, skip link,
 * has-children flag, first source as ints) and the sorted source list. */
ARGOT_B200_API int argot_b200_dev_tree_copy(const argot_b200_dev_tree *d, float *pos4, double *spec64,
                                            int *nodes8, int *src_list, void *stream);

/* ---- light rays --------------------------------------------------------- */

/* Rays are generated per BLOCK of 32 target cells (2 x 4 x 4 cells along
 * x, y, z; lane = lz + 4*ly + 16*lx) by a warp-cooperative walk of the tree
 * with the reference's opening test r^2 theta^2 > L^2
 * (setup_light_ray_tree.c:321-395).  A ray is one 32-bit word
 * (emitter << 5) | lane; a block's rays are contiguous, and the rays of one
 * target cell appear in the reference's depth-first order.
 * blk_offsets: nblocks+1 uint64 prefix offsets.  Blocks cover the local
 * mesh in (bx, by, bz) order with bz fastest; cells outside the mesh in a
 * partial block have no rays. */
ARGOT_B200_API int argot_b200_num_blocks(const argot_b200_grid *g, uint64_t *nblocks);

/* Pass 1: ray counts per block (blk_count: nblocks uint64) for blocks
 * [b0, b1); optional per-cell counts (cell_count: ncell uint32, may be
 * NULL). */
ARGOT_B200_API int argot_b200_count_rays(const argot_b200_grid *g, const argot_b200_dev_tree *t,
                          uint64_t b0, uint64_t b1, uint64_t *blk_count_dev,
                          uint32_t *cell_count_dev, void *stream);
/* exclusive prefix sum of blk_count[b0,b1) into blk_offsets[b0..b1] (device),
 * starting at base; also returns the total on the host if total != NULL. */
ARGOT_B200_API int argot_b200_scan_blocks(const uint64_t *blk_count_dev, uint64_t nb, uint64_t base,
                           uint64_t *blk_offsets_dev, uint64_t *total, void *stream);
/* The same scan, allocating no memory: for callers that cannot allocate
 * device memory while the path runs (hosts that give all device memory to
 * their own pool allocator up front, drop-in callers whose host code forbids
 * cudaMalloc after start-up, loops that must not wait on the driver's
 * allocator).  No
 * counterpart in the reference.  Its scratch is a fixed 64 KiB device array
 * that every GPU loading the library holds until exit: nb is limited to
 * 16 777 216 blocks (larger requests return ARGOT_B200_EINVAL and launch
 * nothing).  All calls on a device share that array, so calls that overlap
 * on the GPU race; serialise them.  The first call on a device looks up the
 * array's address: make it before any stream capture.  With total != NULL
 * the call copies the total back and synchronises `stream`; with NULL it
 * only enqueues work, and blk_offsets[nb] holds the total on the device. */
ARGOT_B200_API int argot_b200_scan_blocks_static(const uint64_t *blk_count_dev, uint64_t nb,
                                                 uint64_t base, uint64_t *blk_offsets_dev,
                                                 uint64_t *total, void *stream);
/* Pass 2: write the ray words of blocks [b0, b1) at blk_offsets[b] - base.
 * A block whose rays do not fit in [blk_offsets[b], blk_offsets[b + 1])
 * (offsets counted for another tree or opening angle) writes only those
 * that fit and sets the device error flag. */
ARGOT_B200_API int argot_b200_emit_rays(const argot_b200_grid *g, const argot_b200_dev_tree *t,
                         uint64_t b0, uint64_t b1, const uint64_t *blk_offsets_dev,
                         uint64_t base, uint32_t *rays_dev, void *stream);

/* ---- march + stitch ----------------------------------------------------- */

#define ARGOT_B200_PRECISION_REFERENCE 0  /* reference FP32 order, bit-exact */
#define ARGOT_B200_PRECISION_KAHAN 1      /* parametric FP32, Kahan columns  */

/* March every ray of blocks [b0, b1): columns (code units) of HI, HeI, HeII
 * from the ray's start (the emitter, clipped to the box as in
 * calc_ray_segment.c:107-126) to the target cell centre.  tau_dev: 3 floats
 * per ray, SoA planes of length nray_group (tau[s*nray_group + r], r
 * relative to base).  crossings (optional, device uint64[1]) receives the
 * number of ray-cell crossings. */
ARGOT_B200_API int argot_b200_march_rays(const argot_b200_grid *g, const void *packed_dev,
                          const argot_b200_dev_tree *t, uint64_t b0, uint64_t b1,
                          const uint64_t *blk_offsets_dev, uint64_t base,
                          const uint32_t *rays_dev, uint64_t nray_group, float *tau_dev,
                          int precision, unsigned long long *crossings_dev,
                          void *stream);

/* March explicit segments (pos6: xs,ys,zs,xe,ye,ze per segment, device) to
 * tau3 (3 floats per segment, AoS).  The drop-in march uses the same
 * kernels. */
ARGOT_B200_API int argot_b200_march_segments(const argot_b200_grid *g, const void *packed_dev,
                              uint64_t nseg, const float *pos6_dev, float *tau3_dev,
                              int precision, void *stream);

/* Stitch: ray_tau[r] = sum of seg_tau over the segments with ray_indx == r
 * (segments sorted by ray index; Kahan-compensated segmented sums).  On one
 * rank, where each ray has one segment per domain, this is the reference's
 * accum_optical_depth. ray_tau3 is AoS (3 floats per ray) and overwritten.
 * A segment whose ray index is >= nray is skipped and sets the device error
 * flag (argot_b200_check_device_error). */
ARGOT_B200_API int argot_b200_stitch(uint64_t nseg, const uint64_t *ray_indx_dev,
                      const float *seg_tau3_dev, uint64_t nray, float *ray_tau3_dev,
                      void *stream);

/* ---- photo-ionisation / heating rates ----------------------------------- */

#define ARGOT_B200_RATE_EXACT_F64 0   /* reference algorithm in FP64        */
#define ARGOT_B200_RATE_EXACT_F32 1   /* FP32, FP64 only for small-dtau phi */
#define ARGOT_B200_RATE_SURROGATE 2   /* BF16 MLP with exact fallback: needs
                                         its weights and workspace, so it runs
                                         through argot_b200_photoion_rays_surrogate;
                                         argot_b200_photoion_rays returns
                                         ARGOT_B200_ENOTSUP for it */

/* Per-cell rates for the target cells of blocks [b0, b1) from their rays'
 * columns.  rates6_dev: 6 planes of ncell floats (Gamma HI, HeI, HeII,
 * Heat HI, HeI, HeII [erg/s]); each cell's sum over its rays is written
 * (mode EXACT_F64 adds to the existing value in ray order with the
 * reference's float rounding, the others overwrite).  Deterministic: no
 * atomics, the rays of a cell are summed in ray order. */
ARGOT_B200_API int argot_b200_photoion_rays(const argot_b200_grid *g, const void *packed_dev,
                             const argot_b200_dev_tree *t, uint64_t b0, uint64_t b1,
                             const uint64_t *blk_offsets_dev, uint64_t base,
                             const uint32_t *rays_dev, uint64_t nray_group,
                             const float *tau_dev, int mode, float *rates6_dev,
                             void *stream);

/* The device fast path of one ray group in one call: optionally the ray
 * generation (emit = 1), then march and rates, the group's blocks [b0, b1)
 * cut into `parts` ranges of about equal ray counts (blk_offsets_host, the
 * host copy of blk_offsets_dev); the march of part p+1 runs on one internal
 * stream while the rates of part p run on another, so the latency-bound
 * march and the SFU-bound rates share the GPU.  rays_dev / tau_dev hold the
 * group's rays from `base` (tau: part p's three column planes start at
 * 3 x its first ray).  The result equals the separate calls bit for bit;
 * `stream` is ordered after all of it (and may be under graph capture). */
ARGOT_B200_API int argot_b200_run_group(const argot_b200_grid *g, const void *packed_dev,
                                        const argot_b200_dev_tree *t, uint64_t b0, uint64_t b1,
                                        const uint64_t *blk_offsets_dev, const uint64_t *blk_offsets_host,
                                        uint64_t base, uint32_t *rays_dev, float *tau_dev, int emit,
                                        int precision, int mode, int parts, float *rates6_dev,
                                        unsigned long long *crossings_dev, void *stream);

/* smooth_photoion_rate (src/smooth_photoion_rate.c:27-1588, single rank):
 * the 27-point smoothing of the six rate planes (layout of rates6 above),
 * centre weighted by 30, normalised by 1/56, in the reference's order and
 * precision (bit-identical); at the mesh faces a copy of the nearest cell
 * (isolated = 1, the reference's default build) or the periodic image
 * (isolated = 0).  out6 must not alias in6. */
ARGOT_B200_API int argot_b200_smooth_rates(const argot_b200_grid *g, const float *in6, float *out6, int isolated,
                                           void *stream);

/* ---- surrogate of the frequency integral (BF16 MLP, tensor cores) ------- */
/* No counterpart in the reference: its unimplemented Gamma(tau) table
 * (multi_freq_bin.h:11-17, prim_chem/calc_gamma_of_tau.c:5-17) is the
 * closest.  The network (4 -> 64 -> 64 -> 64 -> 6, SiLU, BF16 weights and
 * activations, FP32 accumulation) predicts q_j = ln(y_j / ylin_j) of the six
 * thin-cell integrals I_j (Gamma and heating of HI, HeI, HeII), where
 * y_j = ln(I_j / I_j0) and ylin_j = -sum_s tau_s m_js is its exact thin
 * limit, from (log10 tau_HI, log10 tau_HeI, log10 tau_HeII, log10 T). */
typedef struct argot_b200_surrogate argot_b200_surrogate;

/* Marks every emitter whose spectrum is a single-temperature blackbody
 * (src_T[i] > 0: the temperature of source i, <= 0: other spectrum) and
 * uploads each emitter's thin-cell integrals I_j0 and first moments m_js,
 * which the surrogate needs. */
ARGOT_B200_API int argot_b200_dev_tree_set_blackbody(const argot_b200_tree *t, argot_b200_dev_tree *d,
                                                     const float *src_T, void *stream);
ARGOT_B200_API int argot_b200_mlp_num_params(void);
/* normalised blackbody spectra on log10 T = 4 + 1.5 k/(nT-1) (nT x 256) and
 * their thin-cell integrals (nT x 6), host arrays */
ARGOT_B200_API int argot_b200_mlp_spectra(int nT, double *spec, double *i0);
/* n training samples of the exact quadrature on the device: X (n x 4),
 * Y (n x 6) = q_j; spec_dev / i0_dev as from argot_b200_mlp_spectra */
ARGOT_B200_API int argot_b200_mlp_samples(const double *spec_dev, const double *i0_dev, int nT, uint64_t n,
                                          uint64_t seed, float *X, float *Y, void *stream);
/* device floats of workspace a training step on nb samples needs */
ARGOT_B200_API uint64_t argot_b200_mlp_workspace(int nb);
/* forward pass (CUDA cores, the training numerics): normalised outputs O
 * (6 x n, output-major); q_j = 3.5 * O - 3.5 */
ARGOT_B200_API int argot_b200_mlp_forward(const float *params, const float *X, int n, float *O, void *stream);
/* one training step (forward, backward, deterministic gradient sums,
 * Adam on the FP32 master parameters); lr == 0 computes the gradient into
 * grad_out without updating */
ARGOT_B200_API int argot_b200_mlp_train_step(float *params, float *m, float *v, const float *X, const float *Y,
                                             int nb, float lr, int step, float *work, float *grad_out,
                                             double *loss_out, void *stream);
/* inference weights on the current device from the FP32 parameters (host),
 * the validated error envelope (6 x 64 bins of predicted q over [-7, 0],
 * bound of |error of q|) and the per-cell relative error budget tol */
ARGOT_B200_API int argot_b200_surrogate_create(const float *params, const float *env, float tol,
                                               argot_b200_surrogate **out);
ARGOT_B200_API void argot_b200_surrogate_free(argot_b200_surrogate *s);
/* the network on raw inputs X (n x 4) with the tensor-core inference
 * numerics: q_j predictions T (n x 6) */
ARGOT_B200_API int argot_b200_surrogate_eval(const argot_b200_surrogate *s, const float *X, int n, float *T,
                                             void *stream);
/* bytes of device workspace argot_b200_photoion_rays_surrogate needs for a
 * ray group of nray_group rays (7 floats per ray) */
ARGOT_B200_API uint64_t argot_b200_surrogate_workspace(uint64_t nray_group);
/* argot_b200_photoion_rays with the surrogate and exact FP32 fallback: per
 * cell and output, the rays whose validated error bounds fit within tol of
 * the cell's total keep the network's prediction, the others take the
 * exact quadrature.  Deterministic.  counters (device uint64[2], optional)
 * receive the numbers of rays taken by the surrogate and by the exact
 * quadrature. */
ARGOT_B200_API int argot_b200_photoion_rays_surrogate(const argot_b200_grid *g, const void *packed_dev,
                                                      const argot_b200_dev_tree *t,
                                                      const argot_b200_surrogate *sur, uint64_t b0, uint64_t b1,
                                                      const uint64_t *blk_offsets_dev, uint64_t base,
                                                      const uint32_t *rays_dev, uint64_t nray_group,
                                                      const float *tau_dev, float *work_dev, float *rates6_dev,
                                                      unsigned long long *counters_dev, void *stream);

/* ---- batching: many problems in one persistent launch -------------------- */
/* No counterpart in the reference, which runs one mesh per process.  Each
 * problem is prepared by the calls above (pack_fields, tree_build +
 * dev_tree_upload, count_rays + scan_blocks, emit_rays over all its blocks
 * with base 0); one launch (fused mode) or one graph of two persistent
 * kernels (split mode) then marches and integrates every ray of every
 * problem (Kahan march + EXACT_F32 rates, the same arithmetic as
 * argot_b200_march_rays + argot_b200_photoion_rays, so each problem's rates
 * equal those of the problem run alone, bit for bit). */
typedef struct argot_b200_batch argot_b200_batch;
typedef struct {
  argot_b200_grid grid;
  const void *packed_dev;                /* argot_b200_pack_fields output */
  const argot_b200_dev_tree *tree;
  const uint64_t *blk_offsets_dev;       /* nblocks + 1, argot_b200_scan_blocks */
  const uint64_t *blk_offsets_host;      /* host copy of the same */
  const uint32_t *rays_dev;              /* every ray of the problem, base 0 */
  float *rates6_dev;                     /* 6 x ncell, overwritten */
} argot_b200_batch_problem;
typedef struct {
  int warps_per_cta;     /* fused mode: 4 or 8 */
  int ctas_per_sm;       /* fused mode: 1..16, 0 = the occupancy limit */
  int blocks_per_item;   /* target blocks per tile of the work queue */
  int order;             /* 0: tiles by estimated cost, largest first; 1: problem order */
  int mode;              /* 0: fused march + rates in one persistent kernel;
                          * 1: split -- a persistent march kernel and a
                          *    persistent rate kernel, columns through HBM
                          *    (12 bytes per ray, allocated on first use), the
                          *    rates of one part overlapping the march of the
                          *    next on a second stream */
  int parts;             /* split mode: 1..64 parts of the tile list */
} argot_b200_batch_config;
/* the problems' device buffers stay owned by the caller and must outlive
 * the batch */
ARGOT_B200_API int argot_b200_batch_create(const argot_b200_batch_problem *problems, int n,
                                           argot_b200_batch **out);
ARGOT_B200_API void argot_b200_batch_free(argot_b200_batch *b);
ARGOT_B200_API int argot_b200_batch_configure(argot_b200_batch *b, const argot_b200_batch_config *cfg);
ARGOT_B200_API int argot_b200_batch_get_config(const argot_b200_batch *b, argot_b200_batch_config *cfg);
ARGOT_B200_API int argot_b200_batch_num_items(const argot_b200_batch *b);
/* one persistent launch over every problem (crossings_dev: optional device
 * counter of ray-cell crossings, added to) */
ARGOT_B200_API int argot_b200_batch_run(argot_b200_batch *b, unsigned long long *crossings_dev, void *stream);
/* the same launch as a CUDA graph, captured on first use (and after every
 * configuration change), replayed on `stream` */
ARGOT_B200_API int argot_b200_batch_graph_launch(argot_b200_batch *b, void *stream);
/* the autotuner: coordinate search over the configuration, each candidate
 * timed with CUDA events over `reps` launches on the batch itself; leaves
 * the fastest configuration set */
ARGOT_B200_API int argot_b200_batch_tune(argot_b200_batch *b, int reps, argot_b200_batch_config *best,
                                         float *best_ms, void *stream);

/* ---- ART diffuse radiation (src/diffuse_photon, one rank) -------------- */
/* Recombination photons along long characteristics in 12 nside^2 HEALPix
 * directions (calc_diffuse_photon_radiation.c, ray_tracing.c,
 * calc_rmesh_data.c, calc_GH_tot.c): per direction every cell of the start
 * face launches a ray, which wraps through the side faces with its
 * intensity reset (one isolated rank) and ends at the far face; the mean
 * over directions of the per-cell ionisation and heating rates is added to
 * the six rate planes. */
typedef struct argot_b200_art argot_b200_art;
/* The reference's angle table for nside (set_angle_info + sort_angle_id,
 * src/diffuse_photon/set_angle.c): dir3[3 n] direction cosines (float, with
 * the +-1e-31 guard), base_corner2[2 n] start face (0..5) and octant, in
 * processing order; corner_count8 (optional) angles per octant.  Returns
 * n = 12 nside^2 (or a negative code). */
ARGOT_B200_API int argot_b200_art_angle_table(int nside, float *dir3, int *base_corner2, int *corner_count8);
/* set_step_func_factor (src/diffuse_photon/set_step_func_factor.c):
 * ionisation and heating factors of HI, HeI, HeII */
ARGOT_B200_API void argot_b200_art_step_factors(float *step6);
/* a direction set on the current device (from argot_b200_art_angle_table or
 * the caller's own table in the same layout) */
ARGOT_B200_API int argot_b200_art_create(const float *dir3, const int *base_corner2, int nang, const float *step6,
                                         argot_b200_art **out);
ARGOT_B200_API void argot_b200_art_destroy(argot_b200_art *a);
ARGOT_B200_API int argot_b200_art_num_angles(const argot_b200_art *a);
/* device workspace bytes for argot_b200_art_rates with angles_per_pass (the
 * workspace must be 32-byte aligned, as cudaMalloc returns it) */
ARGOT_B200_API uint64_t argot_b200_art_workspace(const argot_b200_grid *g, int angles_per_pass);
/* fields8_dev: 8 planes of ncell floats: dens, fHI, fHII, fHeI, fHeII,
 * fHeIII, felec, uene (fluid_mesh dens, prev_chem fractions, prev_uene);
 * uenetok: run_param.uenetok (uene -> T).  ADDS the diffuse rates to
 * rates6_dev (layout of rates6 above).  The grid is one rank covering the
 * box.  crossings_dev (optional) is added the number of ray-cell steps.
 * Device errors (a ray beyond its step bound) are reported by
 * argot_b200_check_device_error. */
ARGOT_B200_API int argot_b200_art_rates(const argot_b200_art *a, const argot_b200_grid *g, double uenetok,
                                        const float *fields8_dev, float *rates6_dev, void *work_dev,
                                        int angles_per_pass, unsigned long long *crossings_dev, void *stream);

/* Replaces src/diffuse_photon/calc_diffuse_photon_radiation.c:37-128 as built
 * with __USE_GPU__ (src/diffuse_photon/diffuse_prototype.h:30) on a single
 * rank: the caller's angle table and step factors (hd_param, filled by its
 * setup_diffuse_photon), the mesh of cuda_mem[0].mesh_dev, whose
 * prev_chem.{Gamma,Heat}{HI,HeI,HeII} receive the diffuse rates (added).
 * mesh, cd_param and this_omp are not used.  Exported by the builds for
 * helium without H2 or the scale factor only. */
struct host_diffuse_param;
struct cuda_diffuse_param;
ARGOT_B200_API void calc_diffuse_photon_radiation(struct fluid_mesh *mesh, struct run_param *this_run,
                                                  struct cuda_mem_space *cuda_mem, struct cuda_param *this_cuda,
                                                  struct host_diffuse_param *hd_param,
                                                  struct cuda_diffuse_param *cd_param, struct omp_param *this_omp);

/* Reads and clears the device-side error flag of the current device (set
 * when a march exceeded its step bound, which only non-finite input can
 * cause, or when a kernel skipped a block whose offsets lie outside
 * [base, base + nray_group] of its call or do not cover the block's rays);
 * synchronises `stream`.  Returns 0 or ARGOT_B200_EDEVICE. */
ARGOT_B200_API int argot_b200_check_device_error(void *stream);

/* frequency grid and cross sections as the reference tabulates them
 * (source.c:38-53, cross_section.c:5-22): nu[256] [nu_L], csect[256x3] */
ARGOT_B200_API void argot_b200_tables(double *nu, float *csect3);
/* photon rate per bin of one source (source.c:104-138): type 0 blackbody
 * (param = T [K]) or 1 power law (param = index) */
ARGOT_B200_API void argot_b200_photon_rate(int type, float param, double total_rate, double *out256);
/* the two integrals that photon rate is formed from: per-bin photon counts
 * of the unnormalised shape and their total over [1, 10^1.5] nu_L; the rate
 * of bin i is counts[i] * (total_rate / norm) */
ARGOT_B200_API void argot_b200_photon_counts(int type, float param, double *counts256, double *norm);

#ifdef __cplusplus
}
#endif
#endif /* ARGOT_B200_H */
