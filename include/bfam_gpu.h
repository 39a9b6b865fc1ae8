/*
 * bfam_gpu.h -- the B200 device layer for bfam's DG elastic hot path.
 *
 * This is the drop-in boundary: plain C, plain pointers and sizes.  It takes
 * the arrays an application already holds in bfam's structs and replaces the
 * reference's OCCA device layer ("bfamo", src/bfam.c:8389-9091,
 * src/bfam.h:1480-1864) for the elastic right-hand side and LSRK step:
 *
 *   reference (bfam)                               here
 *   ----------------------------------------------------------------------
 *   bfam_subdomain_dgx_t: N, K, Np, r, w, Dr,     bfam_gpu_volume_t
 *     vmapM, vmapP (src/bfam.h:1364-1420)
 *   bfam_subdomain_dgx_glue_data_t: EToEp, EToHp,  bfam_gpu_glue_t
 *     EToOp, EToEm, EToFm, EToHm, mapOp,
 *     interpolation[3], projection[3]
 *     (src/bfam.h:1319-1362)
 *   bfam_subdomain_dgx_field_add + field arrays    bfam_gpu_domain_set_fields
 *     (src/bfam.c:6574-6597)                         / _get_fields
 *   bfamo_device_malloc with memory budget         bfam_gpu_domain_create
 *     (src/bfam.c:8561-8589)                         (opts.mem_budget_bytes)
 *   bfamo_lsrk_t / bfamo_lsrk_init                 bfam_ts_lsrk_init
 *     (src/bfam.h:1840-1863, src/bfam.c:8996-9090)
 *   application stage kernels via BFAMO_KERNEL_RUN bfam_ts_lsrk_step
 *     (src/bfam.h:1673-1717)
 *   bfamo_communicator_post_* / *_wait             (none: neighbour traces
 *     (src/bfam.c:8900-8930)                        are read on the device)
 *
 * Every function returns 0 on success and a negative BFAM_GPU_E* code on
 * failure; bfam_gpu_last_error() gives the message.  The library never
 * aborts the process.  One domain is not safe to use from two host threads
 * at once.
 */
#ifndef BFAM_GPU_H
#define BFAM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum
{
  BFAM_GPU_OK = 0,
  BFAM_GPU_EINVAL = -1,   /* malformed input (sizes, maps, operators) */
  BFAM_GPU_ENOMEM = -2,   /* device allocation failed or over budget */
  BFAM_GPU_ECUDA = -3,    /* CUDA runtime error */
  BFAM_GPU_ETIMEOUT = -4, /* a bounded device-side wait gave up */
  BFAM_GPU_EUNSUPPORTED = -5 /* order / dimension not compiled in */
};

/* numerical flux */
enum
{
  BFAM_GPU_FLUX_UPWIND = 0,
  BFAM_GPU_FLUX_CENTRAL = 1
};

/* arithmetic of the right-hand side; state and LSRK stay FP64 either way */
enum
{
  BFAM_GPU_PRECISION_FP64 = 0,
  /* volume derivative, flux, lift and mortar interpolation in FP32; the
   * mortar L2 projection, stage update and energy in FP64 */
  BFAM_GPU_PRECISION_FP32 = 1
};

/* One dgx volume subdomain (bfam_subdomain_dgx_t) of an adapted Cartesian
 * mesh.  Arrays are read during bfam_gpu_domain_create only. */
typedef struct
{
  int dim;          /* 2 or 3 */
  int N;            /* order; Nq = N+1 nodes per axis */
  int32_t K;        /* elements */
  const double *r;  /* Nq LGL nodes (bfam "r_N") */
  const double *w;  /* Nq LGL weights ("w_N") */
  const double *Dr; /* Nq*Nq differentiation matrix ("Dr_N"), column-major */
  const int32_t *vmapM; /* K * 2dim * Nfp */
  const int32_t *vmapP; /* K * 2dim * Nfp */
  /* affine element geometry: lower corner and edge lengths, K*3 each */
  const double *x0;
  const double *h;
  /* isotropic material per element */
  const double *rho;
  const double *lambda;
  const double *mu;
} bfam_gpu_volume_t;

/* The local glue grid holding this subdomain's hanging faces
 * (bfam_subdomain_dgx_glue_data_t; minus and plus side in one subdomain).
 * K == 0 for a conforming mesh. */
typedef struct
{
  int32_t K;
  const int32_t *EToEp;
  const int8_t *EToHp;
  const int8_t *EToOp;
  const int32_t *EToEm;
  const int8_t *EToFm;
  const int8_t *EToHm;
  /* 1-D operators, Nq*Nq column-major; NULL means identity.
   * interpolation: [same, refine-to-bottom, refine-to-top];
   * projection:    [same, coarsen-from-bottom, coarsen-from-top] */
  const double *interpolation[3];
  const double *projection[3];
} bfam_gpu_glue_t;

typedef struct
{
  int flux;              /* BFAM_GPU_FLUX_* */
  int precision;         /* BFAM_GPU_PRECISION_* */
  size_t mem_budget_bytes; /* 0: no budget beyond the device's free memory */
  int device;            /* CUDA device ordinal */
} bfam_gpu_options_t;

/* Boundary faces of a non-periodic mesh: the minus side of bfam's boundary
 * glue subdomain (`_glue_boundary`, src/bfam.c:7851-7899; bfam builds the
 * grid but leaves the condition to the application), one entry per face
 * whose vmapP points to the element itself, with the condition imposed
 * there through the upwind flux against a ghost state:
 *   free surface (traction-free): v+ = v-, S+ n = -S- n  (T* = 0);
 *   absorbing (characteristic):   v+ = 0, S+ = 0 with the same material. */
enum
{
  BFAM_GPU_BC_FREE_SURFACE = 0,
  BFAM_GPU_BC_ABSORBING = 1,
  /* glued to a face of another domain (bfam's glue grid between two volume
   * subdomains, e.g. of different orders): the pair is declared with
   * bfam_gpu_pglue_create and the two domains step in one batch */
  BFAM_GPU_BC_GLUED = 2
};
typedef struct
{
  int32_t K;            /* boundary faces */
  const int32_t *EToE;  /* element of each face */
  const int8_t *EToF;   /* face of that element */
  const int8_t *type;   /* BFAM_GPU_BC_* */
} bfam_gpu_boundary_t;

typedef struct bfam_gpu_domain bfam_gpu_domain_t;
typedef struct bfam_ts_lsrk bfam_ts_lsrk_t;

/* Validate vol/glue, derive the compact on-device neighbour tables from
 * vmapP and the glue arrays, upload geometry, material and operators and
 * allocate the state (q twice, dq).  Fields start at zero. */
int bfam_gpu_domain_create(const bfam_gpu_volume_t *vol,
                           const bfam_gpu_glue_t *glue,
                           const bfam_gpu_options_t *opts,
                           bfam_gpu_domain_t **out);
/* The same with the boundary faces of a non-periodic mesh (bnd may be NULL;
 * then every face must have a neighbour or a glue element). */
int bfam_gpu_domain_create_with_boundary(const bfam_gpu_volume_t *vol,
                                         const bfam_gpu_glue_t *glue,
                                         const bfam_gpu_boundary_t *bnd,
                                         const bfam_gpu_options_t *opts,
                                         bfam_gpu_domain_t **out);

/* Element geometry from p4est quadrant data, computed on the device: the
 * per-element layout bfam's device kernels were given for this purpose
 * (ID_QUAD_TID, ID_QUAD_LVL, ID_QUAD_X/Y/Z, NQUAD and QUAD_ROOT_LEN,
 * src/bfam.h:1600-1606, src/bfam.c:8697-8705).  Element e lies in tree
 * t = quads[NQUAD e + 0] at level l = quads[NQUAD e + 1] with integer lower
 * corner (x, y, z) = quads[NQUAD e + 2 .. 4] in [0, root_len); its box is
 *   x0_a = tree_x0[3 t + a] + tree_h[3 t + a] * (x_a / root_len),
 *   h_a  = tree_h[3 t + a] * 2^-l.
 * Trees are affine boxes (a brick connectivity's trees after the
 * application's coordinate map): tree_x0/tree_h are their lower corners and
 * edge lengths, one row per tree. */
enum
{
  BFAM_GPU_NQUAD = 5
};
typedef struct
{
  int32_t num_trees;
  const double *tree_x0;  /* [num_trees][3] */
  const double *tree_h;   /* [num_trees][3], > 0 on the mesh's axes */
  const int32_t *quads;   /* [K][BFAM_GPU_NQUAD]: tree, level, x, y, z */
  int32_t root_len;       /* P4EST_ROOT_LEN: a power of two, <= 2^30 */
} bfam_gpu_quadrants_t;

/* bfam_gpu_domain_create_with_boundary with the element boxes computed on
 * the device from quads (vol->x0 and vol->h are not read and may be NULL):
 * the host uploads 20 bytes per element instead of 48 and computes no
 * per-element geometry. */
int bfam_gpu_domain_create_from_quadrants(const bfam_gpu_volume_t *vol,
                                          const bfam_gpu_glue_t *glue,
                                          const bfam_gpu_boundary_t *bnd,
                                          const bfam_gpu_quadrants_t *quads,
                                          const bfam_gpu_options_t *opts,
                                          bfam_gpu_domain_t **out);
/* The element boxes the domain computes with: lower corners and edge
 * lengths, [K][3] each (either may be NULL). */
int bfam_gpu_domain_get_geometry(bfam_gpu_domain_t *dom, double *x0,
                                 double *h);
int bfam_gpu_domain_free(bfam_gpu_domain_t *dom);

/* Number of fields (5 in 2D: vx vy sxx syy sxy; 9 in 3D: vx vy vz sxx syy
 * szz sxy sxz syz) and their length K*Np. */
int bfam_gpu_domain_num_fields(const bfam_gpu_domain_t *dom);
size_t bfam_gpu_domain_field_length(const bfam_gpu_domain_t *dom);
/* device bytes held by the domain */
size_t bfam_gpu_domain_device_bytes(const bfam_gpu_domain_t *dom);

/* Copy the state from / to bfam's per-field host arrays (fields[f] holds
 * K*Np doubles, node fastest, element next). Synchronous. */
int bfam_gpu_domain_set_fields(bfam_gpu_domain_t *dom,
                               const double *const *fields);
int bfam_gpu_domain_get_fields(bfam_gpu_domain_t *dom, double *const *fields);

/* Evaluate the right-hand side of the current state into fields (host). */
int bfam_gpu_domain_rhs(bfam_gpu_domain_t *dom, double *const *rhs);

/* Discrete energy sum_e J_e sum_n w_n (rho|v|^2 + S:C^-1:S)/2 (FP64). */
int bfam_gpu_domain_energy(bfam_gpu_domain_t *dom, double *energy);

/* The same energy, computed without allocating any device memory.  No
 * counterpart in the reference (bfam has no energy diagnostic on the device).
 *
 * For callers that cannot allocate: an application that has handed all of the
 * device's memory to its own pool (a serving process that commits its whole
 * HBM budget to admitted solves), or a monitoring hook that runs between time
 * steps of someone else's solve, where a cudaMalloc can fail or stall.
 * bfam_gpu_domain_energy allocates its per-element scratch on first use; this
 * entry point instead uses a fixed scratch array compiled into the library
 * (BFAM_GPU_NOALLOC_MAX_ELEMENTS + 1 doubles, about 2 MB, held on every GPU
 * that loads the library until the process exits) and calls no cudaMalloc,
 * cudaFree or other allocating routine.
 *
 * Limits: domains with more than BFAM_GPU_NOALLOC_MAX_ELEMENTS elements are
 * rejected with BFAM_GPU_EINVAL.  The first call on a device looks up the
 * array's device address for that device; make that first call before any
 * stream capture.  All calls in the process share the one array: two calls
 * whose work overlaps on the GPU (different streams or devices sharing a
 * context) race and may return wrong values -- serialise them.  Every element
 * slot is rewritten by each call, so no clearing is needed between calls. */
/* The address is looked up once per device ordinal and kept for the process:
 * this assumes the device's primary context and no cudaDeviceReset in
 * between. */
#define BFAM_GPU_NOALLOC_MAX_ELEMENTS 262144
int bfam_gpu_domain_energy_noalloc(bfam_gpu_domain_t *dom, double *energy);

/* Device pointer of field f of the current state (for callers that keep
 * inputs resident and time device work only). */
double *bfam_gpu_domain_field_device_ptr(bfam_gpu_domain_t *dom, int f);

/* Stream the domain launches on (cudaStream_t passed as void*; NULL is the
 * legacy default stream).  Work already queued on the previous stream (steps
 * are asynchronous) completes before anything queued on the new one: the new
 * stream waits for the old one's work, without blocking the host.  The
 * domain's device memory is returned to the library's memory pool in stream
 * order on this stream when the domain is freed, so the stream must outlive
 * the domain. */
int bfam_gpu_domain_set_stream(bfam_gpu_domain_t *dom, void *stream);

/* Per-launch timing, the counterpart of the reference's KERNEL_TIME hook
 * (BFAMO_KERNEL_RUN accumulating each kernel's time, GB/s and GFLOP/s into
 * sc_statistics, src/bfam.h:1673-1708, src/bfam.c:8428-8475).  With
 * profiling on (enable != 0; off by default) every stage launch of the
 * domain is bracketed by a pair of CUDA events on its stream and steps run
 * eagerly (no graph replay); bfam_gpu_domain_kernel_stats waits for the
 * recorded launches and returns, per launch level (level 0: elements without
 * coarse-side hanging faces), the launches, elements, device milliseconds,
 * algorithmic bytes (FP64 q and dq streams: 32 bytes per DOF and stage, 24 in
 * the first stage, 16 for a right-hand-side evaluation) and their GB/s.
 * Enabling or disabling clears the totals.  Independently of this switch,
 * each bfam_ts_lsrk_step and each LSRK stage is an NVTX range, for timeline
 * tools. */
typedef struct
{
  int level;
  int64_t launches;
  int64_t elements;
  double ms;        /* device time summed over the launches */
  double alg_bytes; /* algorithmic bytes summed over the launches */
  double gbs;       /* alg_bytes / time */
} bfam_gpu_kernel_stat_t;
int bfam_gpu_domain_profile(bfam_gpu_domain_t *dom, int enable);
int bfam_gpu_domain_kernel_stats(bfam_gpu_domain_t *dom,
                                 bfam_gpu_kernel_stat_t *out, int max_levels,
                                 int *nlevels);

/* Domains and batches allocate from a stream-ordered memory pool that the
 * library creates per device and owns (other users of the device's default
 * pool are unaffected).  Freed blocks stay in that pool for the next domain;
 * this returns what it holds unused beyond keep_bytes to the device. */
int bfam_gpu_trim_pool(int device, size_t keep_bytes);

/* LSRK stepper over a domain; method numbering follows bfamo_lsrk_method_t
 * (0 KC54, 1 FE, 2 HEUN, 3 W33). */
int bfam_ts_lsrk_init(bfam_ts_lsrk_t **ts, bfam_gpu_domain_t *dom, int method,
                      double t0);
/* Advance nsteps steps of size dt.  Asynchronous on the domain's stream;
 * use_graph != 0 replays each step from a captured CUDA graph. */
int bfam_ts_lsrk_step(bfam_ts_lsrk_t *ts, double dt, int nsteps,
                      int use_graph);
int bfam_ts_lsrk_time(const bfam_ts_lsrk_t *ts, double *t);
int bfam_ts_lsrk_free(bfam_ts_lsrk_t *ts);

/* Wait for the domain's stream and report device-side errors. */
int bfam_gpu_domain_sync(bfam_gpu_domain_t *dom);

/* Launches per LSRK stage (and per right-hand side): 1 for a conforming
 * mesh; with 2:1 hanging faces one per refinement level, because an element
 * with coarse-side hanging faces sums the projected mortar jumps that the
 * fine elements across those faces produce earlier in the same stage. */
int bfam_gpu_domain_launch_levels(const bfam_gpu_domain_t *dom);

/* ------------------------------------------------------------------------
 * Point source and receivers (the serving requests' solves).  No
 * counterpart in the reference: bfam's DG path has no sources or receivers
 * (its applications supplied their own).  With either present, every LSRK
 * step ends with one post-step launch that samples the receivers and
 * advances the domain's device clock (the source's time base).
 * ---------------------------------------------------------------------- */

/* Ricker-wavelet point force f(t) F, f(t) = (1 - 2a) exp(-a),
 * a = (pi f0 (t - t0))^2, added to the velocity equation as
 * f(t) F phi_n(x) / (rho w_n J) at the nodes n of the element holding x
 * (the point force projected on the Lagrange basis with the lumped LGL
 * mass).  The element holding x is the one whose half-open box
 * [x0, x0 + h) contains it. */
typedef struct
{
  double x[3];     /* location (z ignored in 2D) */
  double force[3]; /* force vector F */
  double f0;       /* peak frequency */
  double t0;       /* time of the peak */
} bfam_gpu_source_t;

/* Set (src != NULL) or remove (NULL) the domain's point source.
 * BFAM_GPU_EINVAL if x lies in no element. */
int bfam_gpu_domain_set_source(bfam_gpu_domain_t *dom,
                               const bfam_gpu_source_t *src);

/* Receivers at nrecv points x[r*3 + a]: after every step each field is
 * interpolated (Lagrange basis of the element holding the point) and stored
 * as sample s of receiver r.  Keeps at most max_samples samples; resets
 * the sample count.  nrecv == 0 removes the receivers. */
int bfam_gpu_domain_set_receivers(bfam_gpu_domain_t *dom, int nrecv,
                                  const double *x, int max_samples);

/* Copy the recorded samples, out[(s*nrecv + r)*num_fields + f], and their
 * count (at most max_samples) into *nsamples.  Synchronises the domain's
 * stream. */
int bfam_gpu_domain_get_seismograms(bfam_gpu_domain_t *dom, double *out,
                                    int *nsamples);

/* ------------------------------------------------------------------------
 * Batches: many independent domains stepped together.  No counterpart in
 * the reference (one bfam domain per MPI rank).  Domains are grouped by
 * (dim, order, precision, flux, operators); each group is one persistent
 * launch per LSRK stage over a flat (domain, element) work list, the groups
 * run on forked streams, and a step is replayed from a CUDA graph.  The
 * domains keep their own state, time step and clock; a domain must not be
 * stepped by another stepper while it belongs to a batch.
 * ---------------------------------------------------------------------- */
typedef struct bfam_gpu_batch bfam_gpu_batch_t;

/* ndom domains on one device; t0[i] is domain i's start time (NULL: each
 * domain keeps the time of its device clock, which starts at 0 and is
 * advanced by every step that has a post-step launch). */
int bfam_gpu_batch_create(bfam_gpu_domain_t *const *doms, int ndom,
                          int method, const double *t0,
                          bfam_gpu_batch_t **out);
/* Launch on this stream (NULL: the batch's own stream); it must outlive the
 * batch (the batch's arrays are freed in stream order on it). */
int bfam_gpu_batch_set_stream(bfam_gpu_batch_t *b, void *stream);
/* Advance every domain nsteps steps, domain i with step dt[i]. */
int bfam_gpu_batch_step(bfam_gpu_batch_t *b, const double *dt, int nsteps,
                        int use_graph);
int bfam_gpu_batch_time(const bfam_gpu_batch_t *b, int i, double *t);
/* Wait for the batch's stream and report device-side errors. */
int bfam_gpu_batch_sync(bfam_gpu_batch_t *b);
/* Kernel launches of one batch step (stage launches of every group and
 * level, plus the post-step launch). */
int bfam_gpu_batch_launches_per_step(const bfam_gpu_batch_t *b);
int bfam_gpu_batch_free(bfam_gpu_batch_t *b);
/* Number of order groups, and group g's (dim, N, precision, elements). */
int bfam_gpu_batch_num_groups(const bfam_gpu_batch_t *b);
int bfam_gpu_batch_group_info(const bfam_gpu_batch_t *b, int g, int *dim,
                              int *N, int *precision, int64_t *elements);

/* ------------------------------------------------------------------------
 * Glue between two domains, e.g. of different orders (p-nonconforming
 * faces): bfam's glue subdomain between two volume subdomains of orders N_m
 * and N_p, whose glue order N_g >= both (src/bfam.c:7340-7414, operators
 * from src/bfam.c:5607-5691 with the N_m != N_p branches at 5656-5667).
 * Each side interpolates its trace to the N_g glue grid, the upwind flux is
 * solved there, and each side's jumps are L2-projected back to its order and
 * lifted by its own element.  The glued faces are the entries of type
 * BFAM_GPU_BC_GLUED in each domain's boundary list; pair k joins entry bm[k]
 * of dm with entry bp[k] of dp: opposite faces (F and F ^ 1) of elements
 * whose boxes meet across them with the same extent along the face, face
 * nodes in the same tangential order (glue orientation 0).  Same-size faces
 * only (a face that is both hanging and of another order is not supported).
 * The coupled domains step together in one batch (bfam_gpu_batch_add_pglue)
 * with the same time step; bfam_ts_lsrk_step and bfam_gpu_domain_rhs refuse
 * a domain with glued faces.
 * ---------------------------------------------------------------------- */
typedef struct
{
  int32_t K;          /* glued face pairs */
  const int32_t *bm;  /* boundary-list entry of each pair in dm */
  const int32_t *bp;  /* boundary-list entry of each pair in dp */
  int N_g;            /* glue order, >= both domains' orders */
  /* glue_m->interpolation[0] / projection[0] of each side: (N_g+1) x (N+1)
   * interpolation to the glue grid and (N+1) x (N_g+1) L2 projection from
   * it, column-major; NULL means identity (only when N == N_g) */
  const double *I_m2g, *P_g2m;
  const double *I_p2g, *P_g2p;
} bfam_gpu_pglue_desc_t;
typedef struct bfam_gpu_pglue bfam_gpu_pglue_t;

int bfam_gpu_pglue_create(bfam_gpu_domain_t *dm, bfam_gpu_domain_t *dp,
                          const bfam_gpu_pglue_desc_t *desc,
                          bfam_gpu_pglue_t **out);
int bfam_gpu_pglue_free(bfam_gpu_pglue_t *g);
/* Step the glue with the batch: one coupling launch per glue and stage,
 * before the stage's element launches.  Both domains must be in the batch;
 * every glued face of the batch's domains must be covered by exactly one
 * added glue when the batch steps. */
int bfam_gpu_batch_add_pglue(bfam_gpu_batch_t *b, bfam_gpu_pglue_t *g);

/* Tile shapes compiled for an order: tile t runs bfam_gpu_tile_elements
 * elements per CTA with `threads` threads each (a tile with fewer threads
 * than nodes or face nodes loops over them; each element of a CTA has its
 * own shared-memory tile and barrier, down to one warp per element) and a
 * register budget for `min_ctas` resident CTAs per SM.  Tile 0 is the
 * single-domain kernel's (one element per CTA). */
int bfam_gpu_tile_count(int dim, int N);
int bfam_gpu_tile_shape(int dim, int N, int tile, int *threads,
                        int *min_ctas);
/* elements per CTA of tile t (>= 1), or a negative BFAM_GPU_E* code */
int bfam_gpu_tile_elements(int dim, int N, int tile);
/* Choose group g's tile and persistent grid (ctas_per_sm CTAs per SM; 0:
 * as many as fit). */
int bfam_gpu_batch_set_tile(bfam_gpu_batch_t *b, int g, int tile,
                            int ctas_per_sm);

/* Kernel launches issued by this library since process start. */
uint64_t bfam_gpu_launch_count(void);

/* Copy of the last error message of the calling thread (NUL-terminated,
 * truncated to len). Returns the message length. */
int bfam_gpu_last_error(char *buf, size_t len);

/* Record msg as the calling thread's last error and return code: for code
 * layered on this C-ABI (the header-only adapter from bfam's objects,
 * include/bfam_gpu_bfam.h) so that its failures read like the library's. */
int bfam_gpu_record_error(int code, const char *msg);

#ifdef __cplusplus
}
#endif
#endif
