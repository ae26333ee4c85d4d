/*
 * terawarp_b200.h -- C ABI of the B200-native TeraWarp warp path.
 *
 * Plain C types only (pointers, sizes, PODs): a caller links
 * libterawarp_b200.so and needs no CUDA, torch or Qt headers.  CUDA streams
 * are passed as opaque `void*` (a cudaStream_t, or NULL for the library's
 * own stream).
 *
 * Every function returns a tw_status.  Nothing here ever calls
 * cudaDeviceReset() (the reference's GPU wrappers do, e.g. chazhi.cu:661);
 * the GPU is shared with the caller.
 *
 * Coordinate conventions (same as the reference):
 *   - volumes are x-fastest, then y, z, channel; sz[4] = {x, y, z, channels}
 *   - warps are pull-back: every output voxel p samples the subject volume
 *     at q(p); a sample with any q_i < 0 or q_i > sz_i - 1 writes 0
 *   - TPS output is (T)(trilinear + 0.5), affine output is (T)(trilinear)
 *   - voxel types: uint8 (the reference's only type) and uint16
 */
#ifndef TERAWARP_B200_H
#define TERAWARP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TW_ABI_VERSION 1

typedef enum {
    TW_OK = 0,
    TW_ERR_ARG = 1,         /* invalid argument (sizes, counts, modes)         */
    TW_ERR_SINGULAR = 2,    /* degenerate landmarks: rank-deficient [1 s] or non-SPD system */
    TW_ERR_OOM = 3,         /* device/pinned allocation failed or over the HBM budget */
    TW_ERR_CUDA = 4,        /* a CUDA runtime call failed                       */
    TW_ERR_TIMEOUT = 5,     /* a bounded wait gave up                           */
    TW_ERR_IO = 6,          /* a tile-source or tile-sink callback failed       */
    TW_ERR_UNSUPPORTED = 7, /* valid request the library does not implement     */
    TW_ERR_NOT_READY = 8    /* asynchronous job not finished yet                */
} tw_status;

typedef enum { TW_U8 = 1, TW_U16 = 2 } tw_dtype;
typedef enum { TW_INTERP_TRILINEAR = 0, TW_INTERP_NEAREST = 1 } tw_interp;

/* One landmark, in voxel coordinates of its image (Coord3D_JBA,
 * q_littleQuickWarp_common.h:12-18; Vaa3D ImageMarker x,y,z). */
typedef struct { float x, y, z; } tw_marker;

typedef struct tw_ctx tw_ctx;   /* device, streams, pinned staging, HBM budget */
typedef struct tw_tps tw_tps;   /* solved TPS coefficients, device-resident     */

/* ---------------------------------------------------------------- context */

/* Creates a context on CUDA device `device`.  hbm_budget_bytes caps what the
 * context allocates on the device (0 = 90% of free memory at creation).
 * No counterpart in the reference, which allocates and resets per call. */
tw_status tw_ctx_create(int device, size_t hbm_budget_bytes, tw_ctx **out);
tw_status tw_ctx_destroy(tw_ctx *ctx);
/* Text of the last error recorded on this context (never NULL). */
const char *tw_ctx_last_error(const tw_ctx *ctx);
const char *tw_status_string(tw_status s);
int tw_abi_version(void);
/* Number of kernels this context has launched (counter for benchmarks). */
uint64_t tw_ctx_kernel_launches(const tw_ctx *ctx);
/* Bytes the context's streaming paths (whole-volume slabs, tiled engine)
 * have copied host -> device and device -> host (counters for benchmarks). */
void tw_ctx_transfer_bytes(const tw_ctx *ctx, uint64_t *h2d, uint64_t *d2h);
/* Blocks until all work queued on the context's streams has finished. */
tw_status tw_ctx_synchronize(tw_ctx *ctx);

/* ------------------------------------------------------ (a) TPS solve FP64 */

/* Solves the regularised TPS system in FP64 on the GPU:
 *   c = q2 (q2' K q2 + lambda I)^-1 q2' Y,   d = r^-1 q1' (Y - K c)
 * with K_ij = -|s_i - s_j|, X = [1 s] = q1 r, Y = [1 t].  `centres` are the
 * TPS kernel centres s (target-image landmarks), `values` the mapped points t
 * (subject-image landmarks), n >= 4.  The reference solves the same system
 * in compute_df_stps_subsampled_volume_4bspline
 * (q_imgwarp_tps_quicksmallmemory.cpp:377-588, FP64 CPU :554-586, FP32 GPU
 * via qr.cu:8, extendornormal.cu:55, GET_A_i.cu:80, aff.cu:37) and in its
 * tiled twin _per (:906-1082).  lambda = 0.2 in the reference (:581).
 * Returns TW_ERR_SINGULAR for coplanar/degenerate centres. */
tw_status tw_tps_solve(tw_ctx *ctx, const tw_marker *centres, const tw_marker *values, int n,
                       double lambda, tw_tps **out);
tw_status tw_tps_destroy(tw_tps *tps);
int tw_tps_count(const tw_tps *tps);
/* Copies the FP64 coefficients to host memory: c is n x 4 row-major
 * (xnx4_c), d is 4 x 4 row-major (x4x4_d). */
tw_status tw_tps_get_coeffs(const tw_tps *tps, double *c, double *d);

/* ---------------------------------------- (b) TPS at the control-grid nodes */

/* Evaluates the displacement f(p) - p at every node of a control grid of
 * gsz0 x gsz1 x gsz2 nodes, node (i,j,k) at ((i-1)g+ox, (j-1)g+oy, (k-1)g+oz),
 * in FP32 with compensated landmark sums.  `dev_nodes` is device memory of
 * gsz0*gsz1*gsz2 float4 (dx, dy, dz, 0), x fastest.  Replaces
 * gpu_computedistance / get_cd (weiyijisuan.cu:91-219) and the CPU loops at
 * q_imgwarp_tps_quicksmallmemory.cpp:620-648 and :1117-1146. */
tw_status tw_tps_eval_grid(tw_ctx *ctx, const tw_tps *tps, int64_t gsz0, int64_t gsz1, int64_t gsz2,
                           int g, int64_t ox, int64_t oy, int64_t oz, void *dev_nodes, void *stream);
/* Grid size rule gsz = ceil(sz/g) + 3 (q_imgwarp_tps_quicksmallmemory.cpp:592). */
int64_t tw_grid_size(int64_t sz, int g);

/* ------------------- (b)+(c) fused B-spline expansion + trilinear resample */

/* Warps a device-resident volume with a device-resident node grid
 * (from tw_tps_eval_grid with ox=oy=oz=0): for every output voxel the cubic
 * B-spline of the 4x4x4 surrounding nodes gives the displacement, then the
 * subject is sampled trilinearly (+0.5, truncation) or by nearest neighbour.
 * src and dst have the same dims sz[0..2] (one channel; call per channel).
 * g must be 4, 8, 16, 32 or 64.  Replaces gpu_interpolation_stps /
 * get_Displacement_brightness_stps (chazhi.cu:226-338, :844-1039) and the
 * CPU loops q_dfblcokinterp_bspline + q_imgblockwarp
 * (q_imgwarp_tps_quicksmallmemory.cpp:85-203). */
tw_status tw_warp_tps_device(tw_ctx *ctx, const void *dev_nodes, int g, int dtype, int interp,
                             const void *dev_src, void *dev_dst, const int64_t sz[3], void *stream);

/* ------------------------------- (d) affine, rotation, translation, scaling */

/* Fits the 4x4 affine T with sub = T tar from n >= 4 landmark pairs (3-D DLT
 * with Hartley normalisation, FP64 on the GPU).  Replaces
 * q_affine_compute_affinmatrix_3D (q_warp_affine_tps.cpp:649-731). M is
 * row-major 4x4 and maps target (output) voxel coordinates to subject
 * coordinates. */
tw_status tw_fit_affine(tw_ctx *ctx, const tw_marker *tar, const tw_marker *sub, int n, double M[16]);

/* Largest n accepted by tw_fit_affine_noalloc. */
#define TW_FIT_AFFINE_NOALLOC_MAX 4096

/* tw_fit_affine without allocating: no device memory is allocated, and on the
 * host nothing but the message of a failed call.  No counterpart in the
 * reference: it exists for callers that cannot allocate at the time they
 * fit, e.g. a process whose device memory is wholly reserved by its own
 * volume cache or by this context's HBM budget (tw_fit_affine would then fail
 * with TW_ERR_OOM), or a loop that must not let an allocation wait on, or
 * stall, warps running on other streams.
 *
 * Its scratch is one fixed array in device memory per device (about 288 KiB,
 * reserved by the CUDA driver when it loads this entry point's device code on
 * that device), so n is limited to TW_FIT_AFFINE_NOALLOC_MAX; larger n
 * returns TW_ERR_ARG.
 * Same kernel, same FP64 arithmetic and same result as tw_fit_affine.
 * Calls that overlapped on the GPU would race on that one array, so calls for
 * the same device are serialised by a lock inside the library, which is held
 * until ctx's stream has finished the call's work (on error returns too).
 * The first call on each device looks up the array's address (and may load
 * the device code); make it before any stream capture begins.  The lookup is
 * repeated when the device's context was destroyed and created again since
 * (cudaDeviceReset), because the array then lives at a new address.
 * Synchronises ctx's stream; the caller's current device is unchanged on
 * return. */
tw_status tw_fit_affine_noalloc(tw_ctx *ctx, const tw_marker *tar, const tw_marker *sub, int n, double M[16]);

/* Builds the pull-back matrix of the TeraWarp command's parameter surface
 * (README.md:85-100), for which the reference source has no code:
 *   warp_mode 0 (non-rigid), deformation_mode 2 (scaling): para = per-axis
 *     scale factors s (0.1..10); the output is the input scaled by s about
 *     the origin voxel, M = diag(1/s).
 *   warp_mode 1 (rigid), deformation_mode 0 (rotation): para = angles in
 *     degrees (-180..180) about x, y, z, applied x then y then z, about the
 *     centre of the input volume ((sz-1)/2), which stays at the centre of the
 *     output volume; M = inverse of that map.
 *   warp_mode 1, deformation_mode 1 (translation): para = step in voxels;
 *     out(p) = in(p - t), M = [I | -t].
 * in_sz / out_sz are the input and output dims (out = in unless resized). */
tw_status tw_make_affine(int warp_mode, int deformation_mode, const double para[3],
                         const int64_t in_sz[3], const int64_t out_sz[3], double M[16]);

/* Warps a device-resident volume with the 4x4 matrix M (FP32 per voxel,
 * truncation).  Output dims may differ from the source (resize).  Replaces
 * gpu_interpolation_affine / get_Displacement_affine (aff.cu:379-447,
 * :539-620) and the OpenMP loop q_warp_affine_tps.cpp:1373-1437. */
tw_status tw_warp_affine_device(tw_ctx *ctx, const double M[16], int dtype, int interp,
                                const void *dev_src, const int64_t src_sz[3],
                                void *dev_dst, const int64_t dst_sz[3], void *stream);

/* ---------------------------------------------- operator-level entry points */

/* Mirror of imgwarp_smallmemory_image (q_imgwarp_tps_quicksmallmemory.h:89-90,
 * body q_imgwarp_tps_quicksmallmemory.cpp:1997-2162) with the same argument
 * order and meaning: ql_marker_tar become the TPS values, ql_marker_sub the
 * TPS centres (the plugin passes subject markers first,
 * plugin_Bigimagewarp.cpp:197).  szBlock_* is the B-spline grid spacing
 * (must be equal, as the reference requires for interp_df = 1, and smaller
 * than the image).  interp_df must be 1 (B-spline; the reference's 0 =
 * linear DF is not on its live path).  interp_img 0 = trilinear, 1 = NN.
 * img_sub / img_warp are caller-owned buffers of sz[0]*sz[1]*sz[2]*sz[3]
 * voxels, host (pinned or pageable) or device; host buffers are streamed
 * through the GPU in z-slabs with H2D, compute and D2H overlapped.
 * The output is returned in img_warp instead of being saved to a file. */
tw_status tw_imgwarp_smallmemory_image(tw_ctx *ctx, const tw_marker *ql_marker_tar,
                                       const tw_marker *ql_marker_sub, int n,
                                       int64_t szBlock_x, int64_t szBlock_y, int64_t szBlock_z,
                                       int interp_df, int interp_img, int dtype,
                                       const void *img_sub, const int64_t sz_img_sub[4], void *img_warp);

/* Mirror of q_imagewarp_affine_image (q_warp_affine_tps.h:74, body
 * q_warp_affine_tps.cpp:1332-1469): fits sub = T tar and warps. */
tw_status tw_q_imagewarp_affine_image(tw_ctx *ctx, const tw_marker *ql_marker_tar,
                                      const tw_marker *ql_marker_sub, int n, int dtype,
                                      const void *img_sub, const int64_t sz_img_sub[4], void *img_out);

/* ----------------------------------------------- (e) tiled out-of-core path */

/* Tile source: copy the source box [x0,x0+nx) x [y0,y0+ny) x [z0,z0+nz)
 * (always inside the volume) into dst (x fastest, row pitch nx, slice pitch
 * nx*ny voxels).  Return 0 on success.  Replaces the per-Z-slice reads of
 * read_2Dtif_BLOCK (Bigwarp.cpp:66-175). */
typedef int (*tw_read_box_fn)(void *user, int64_t x0, int64_t y0, int64_t z0,
                              int64_t nx, int64_t ny, int64_t nz, void *dst);
/* Tile sink: receives one finished output tile (x fastest, pitch nx, nx*ny).
 * Return 0 on success.  Replaces the per-tile saveImage of
 * q_imgwarp_tps_quicksmallmemory.cpp:1863-1884. */
typedef int (*tw_write_box_fn)(void *user, int64_t x0, int64_t y0, int64_t z0,
                               int64_t nx, int64_t ny, int64_t nz, const void *src);

/* An in-memory volume (x fastest) served by the two functions below.  When
 * `data` is pinned host memory (cudaHostAlloc / cudaHostRegister), the tiled
 * entry points recognise these functions and move boxes with strided DMA
 * copies instead of calling them.  threads: host threads for the copy
 * (0 = half the cores). */
typedef struct {
    void *data;
    int64_t sz[3];
    int dtype;
    int threads;
} tw_host_volume;
/* tw_read_box_fn over a tw_host_volume (user = tw_host_volume*). */
int tw_box_reader_host(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                       void *dst);
/* tw_write_box_fn over a tw_host_volume (user = tw_host_volume*). */
int tw_box_writer_host(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                       const void *src);

/* A procedural volume for running the tiled path at terabyte scale with no
 * stored volume: every voxel is a function of its coordinates and the seed
 * (hash noise 0..10, Gaussian blobs, short random-walk fibres), so any two
 * boxes agree where they overlap.  threads: host threads per box (0 = all). */
typedef struct {
    uint64_t seed;
    int64_t sz[3];
    int dtype;
    int threads;
} tw_synthetic_volume;
/* tw_read_box_fn over a tw_synthetic_volume (user = tw_synthetic_volume*). */
int tw_box_reader_synthetic(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                            void *dst);

/* A sink that keeps only a checksum of what it receives: the sum of the
 * voxel values, a position-weighted sum (a tile written to the wrong place
 * changes it), and the voxel count.  Zero-initialise before use. */
typedef struct {
    uint64_t sum, weighted, voxels;
    int dtype;
    int threads;
} tw_checksum;
/* tw_write_box_fn over a tw_checksum (user = tw_checksum*). */
int tw_box_writer_checksum(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                           const void *src);

typedef struct {
    int64_t tile[3];        /* output tile dims x, y, z (0 = 512; reference:    */
                            /* 1000^3); TPS tiles are rounded down to whole     */
                            /* resample units (64 x 16 x g), at least one unit  */
    int staging_depth;      /* tiles in flight, 2..4 (0 = 2: double buffering)  */
    int interp;             /* tw_interp                                        */
    int64_t region_o[3];    /* output region to warp: [region_o, region_o +     */
    int64_t region_n[3];    /* region_n) (all region_n 0 = the whole output);   */
                            /* the sink receives only tiles of it.  A TPS       */
                            /* region grows to whole resample units (64 x 16 x  */
                            /* g voxels of the output grid)                     */
} tw_tile_opts;

/* Mirror of imgwarp_smallmemory_CYF (q_imgwarp_tps_quicksmallmemory.h:86-87,
 * body :1161-1994) for volumes larger than the GPU: solves once, keeps the
 * node grid device-resident, and streams output tiles through pinned
 * double-buffered transfers on separate copy/compute streams.  Each tile's
 * source box is the exact footprint of its samples (convex-hull bound of the
 * B-spline) and tiles start on the whole volume's brick boundaries, so the
 * tiled result equals the whole-volume result voxel for voxel.
 * marker_scale multiplies both marker sets (the reference uses 4 for markers
 * placed on a 4x downsampled image, :1194-1203). */
tw_status tw_imgwarp_smallmemory_tiled(tw_ctx *ctx, const tw_marker *ql_marker_tar,
                                       const tw_marker *ql_marker_sub, int n, double marker_scale,
                                       int g, int dtype, const int64_t sz[3],
                                       tw_read_box_fn read_box, void *read_user,
                                       tw_write_box_fn write_box, void *write_user,
                                       const tw_tile_opts *opts);

/* A (tile shape, staging depth) candidate of the tiled TPS path and the time
 * the tuner measured for it (seconds; filled in by tw_tune_tiled_tps). */
typedef struct {
    int64_t tile[3];
    int staging_depth;
    double seconds;
} tw_tile_candidate;

/* Chooses the tile shape and staging depth of tw_imgwarp_smallmemory_tiled
 * for one job by timing the candidates (cands/ncands, or a built-in list when
 * cands is NULL; times are written back into cands) on the job's corner block
 * (sample dims x, y, z; 0 = 1024 x 1024 x 512, clipped to the volume): the
 * job's own landmarks are solved and its node grid evaluated once, then each
 * candidate streams the sample through the tiled engine from read_box into a
 * sink that discards it.  The choice is remembered per (volume dims, dtype,
 * g, landmark-count power-of-two bucket, device name) for the process, and
 * in cache_path when it is given (a text file of "key tx ty tz depth seconds"
 * lines, the last line of a key winning).  best receives the chosen tile and
 * depth (interp 0, whole volume).  With ctx NULL only the cache file is
 * consulted (TW_ERR_NOT_READY on a miss).  No counterpart in the reference,
 * whose tiles are 1000^3 (q_imgwarp_tps_quicksmallmemory.cpp:1264). */
tw_status tw_tune_tiled_tps(tw_ctx *ctx, const tw_marker *ql_marker_tar, const tw_marker *ql_marker_sub, int n,
                            double marker_scale, int g, int dtype, const int64_t sz[3], tw_read_box_fn read_box,
                            void *read_user, tw_tile_candidate *cands, int ncands, const int64_t sample[3],
                            const char *cache_path, tw_tile_opts *best);

/* Mirror of q_imagewarp_affine_cyf (q_warp_affine_tps.h:72, body :851-1329)
 * for an arbitrary matrix: output dims out_sz, tiles streamed as above. */
tw_status tw_warp_affine_tiled(tw_ctx *ctx, const double M[16], int dtype, const int64_t src_sz[3],
                               const int64_t out_sz[3], tw_read_box_fn read_box, void *read_user,
                               tw_write_box_fn write_box, void *write_user, const tw_tile_opts *opts);

/* ------------------------------------------- plugin-level parameter surface */

/* The TeraWarp command's parameters (README.md:85-100) plus the constants the
 * reference hard-codes.  device_mode must be 1: there is no CPU path here. */
typedef struct {
    int warp_mode;          /* 0 non-rigid, 1 rigid                                  */
    int device_mode;        /* must be 1 (GPU)                                       */
    int resize_mode;        /* 1: output dims = newsize_*                            */
    int deformation_mode;   /* warp_mode 0: 0 affine, 1 TPS, 2 scaling;
                               warp_mode 1: 0 rotation, 1 translation                */
    double para_x, para_y, para_z;
    int64_t newsize_x, newsize_y, newsize_z;
    int grid_spacing;       /* B-spline control spacing (0 = 4, plugin_Bigimagewarp.cpp:197) */
    double marker_scale;    /* 0 = 1.0 (whole image); the reference's tiled path uses 4 */
    double lambda;          /* 0 = 0.2 (q_imgwarp_tps_quicksmallmemory.cpp:581)       */
    int interp;             /* tw_interp                                              */
    int downsample_mode;    /* 1: also write a downsampled preview of the result
                               (the plugin's downsample_mode,
                               plugin_Bigimagewarp.cpp:93, :264-325; used by
                               tw_bigimagewarp_files)                                 */
} tw_params;

/* Fills *p with the reference's defaults (TPS, GPU, spacing 4, lambda 0.2). */
void tw_params_default(tw_params *p);

/* Output dims the call below produces for input dims in_sz. */
tw_status tw_output_size(const tw_params *p, const int64_t in_sz[3], int64_t out_sz[3]);

/* Plugin-level warp of an in-memory volume (bigimagewarp,
 * plugin_Bigimagewarp.cpp:123-336, whole-image branch): dispatches affine /
 * TPS / scaling / rotation / translation, with optional resize.  marker_sub /
 * marker_tar are the subject and target landmark files' contents (used by
 * affine and TPS).  img_out must hold the tw_output_size dims x sz[3]. */
tw_status tw_bigimagewarp(tw_ctx *ctx, const tw_params *p, const tw_marker *marker_sub,
                          const tw_marker *marker_tar, int n, int dtype, const void *img_sub,
                          const int64_t sz[4], void *img_out);

/* Downsample preview of q_imagewarp_affine_cyf_downsample
 * (q_warp_affine_tps.cpp:1474-1519): factor = round-half-up(maxdim / 600),
 * at least 1; output dims sz / factor. */
int tw_downsample_factor(const int64_t sz[3]);
tw_status tw_downsample_image(tw_ctx *ctx, int dtype, const void *img, const int64_t sz[4],
                              void *img_out, int64_t out_sz[3]);

/* ------------------------------------------------------------------- files */

/* Vaa3D raw stacks (.v3draw, and the .raw slice files of the tiled path), as
 * the reference reads them in loadMetadata_cyf (RawFmtMngr.cpp:332-446) and
 * writes them in saveStack2Raw_cyf (Bigwarp.cpp:660-751): the 24-byte key
 * "raw_image_stack_by_hpeng", one endianness byte ('L' or 'B'), a 2-byte data
 * type code (bytes per voxel: 1, 2 or 4), four 4-byte sizes x, y, z,
 * channels, then the voxels, x fastest.  Files of either byte order are
 * read; files are written in the host's order.  dtype is TW_U8, TW_U16, or 4
 * for a float32 stack (readable, not warpable).  These functions use no GPU. */
tw_status tw_v3draw_read_header(const char *path, int64_t sz[4], int *dtype, int64_t *header_bytes);
/* Reads the whole payload (every channel) into dst (dst_bytes at least
 * x*y*z*channels*bytes per voxel). */
tw_status tw_v3draw_read(const char *path, void *dst, size_t dst_bytes);
/* Reads box [x0,x0+nx) x [y0,y0+ny) x [z0,z0+nz) of channel 0 into dst (x
 * fastest, pitch nx, nx*ny); replaces copyRawFileBlock2Buffer_cyf
 * (RawFmtMngr.cpp:1511-1695), with one positioned read per row run. */
tw_status tw_v3draw_read_box(const char *path, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny,
                             int64_t nz, void *dst);
tw_status tw_v3draw_write(const char *path, const void *data, const int64_t sz[4], int dtype);

/* A directory of per-Z raw slice files (one x*y plane each) as a tile source:
 * the files are every entry but ".", "..", "mdata.bin" and ".iim.format",
 * sorted by name, one per z (read_2Dtif_dir, dir_make.cpp:175-216); all must
 * share plane size and type.  threads: planes read in parallel (0 = up to
 * 16).  Replaces read_2Dtif_BLOCK (Bigwarp.cpp:66-175). */
typedef struct tw_slice_dir tw_slice_dir;
tw_status tw_slice_dir_open(const char *dir, int threads, tw_slice_dir **out);
tw_status tw_slice_dir_info(const tw_slice_dir *d, int64_t sz[3], int *dtype);
tw_status tw_slice_dir_close(tw_slice_dir *d);
/* tw_read_box_fn over a tw_slice_dir (user = tw_slice_dir*). */
int tw_box_reader_slices(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                         void *dst);

/* A tile sink that writes finished output tiles straight into per-Z raw
 * slice files in `dir` (created if needed), named as the reference names its
 * stitched output: "%07d.raw" of z * 10 (saveImage_PJ, Bigwarp.cpp:957-1004).
 * Every slice file is created at its full size by tw_slice_writer_create, so
 * tiles may arrive in any order; this replaces saving tiles and stitching
 * them into slices in a second pass (Bigwarp.cpp:229-573, :958-1121). */
typedef struct tw_slice_writer tw_slice_writer;
tw_status tw_slice_writer_create(const char *dir, const int64_t sz[3], int dtype, int threads,
                                 tw_slice_writer **out);
tw_status tw_slice_writer_close(tw_slice_writer *w);
/* tw_write_box_fn over a tw_slice_writer (user = tw_slice_writer*). */
int tw_box_writer_slices(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                         const void *src);

/* Vaa3D .marker files (read by readMarker_file, plugin_Bigimagewarp.cpp:145):
 * comma-separated lines "x,y,z,radius,shape,name,comment,r,g,b"; lines that
 * start with '#' and lines without three leading numbers are skipped.  x, y, z
 * are returned as written (the plugin passes them to the warp unchanged).
 * With out = NULL only *n is set; otherwise capacity must hold *n markers. */
tw_status tw_marker_file_read(const char *path, tw_marker *out, int capacity, int *n);
tw_status tw_marker_file_write(const char *path, const tw_marker *m, int n);

/* The plugin's whole command on files (bigimagewarp,
 * plugin_Bigimagewarp.cpp:123-336): reads the two marker files, then
 *   - img_sub a .v3draw file: warps it in memory (tw_bigimagewarp) and writes
 *     out_dir/<name><suffix>.v3draw;
 *   - img_sub a directory of slices: warps it tile by tile from the slices
 *     into out_dir/<name><suffix>_slice/ (slice files, written as tiles finish);
 * with suffix _affine, _stps, _scaling, _rotation or _translation by mode.
 * downsample_mode 1 also writes the downsampled preview (factor
 * tw_downsample_factor) as <name><suffix>_downsample.v3draw or
 * <name><suffix>_downsample_slice/.  marker_scale 0 means the reference's
 * choice: 1 for a .v3draw, 4 for a slice directory
 * (q_imgwarp_tps_quicksmallmemory.cpp:1194-1203, q_warp_affine_tps.cpp:866-874). */
tw_status tw_bigimagewarp_files(tw_ctx *ctx, const tw_params *p, const char *img_sub, const char *marker_sub,
                                const char *marker_tar, const char *out_dir);

/* ------------------------------------------------------------- serving loop */

typedef struct tw_server tw_server;

typedef struct {
    int kind;               /* 0 affine (matrix), 1 TPS (landmarks)                  */
    int dtype;              /* tw_dtype                                              */
    int interp;             /* tw_interp                                             */
    int g;                  /* TPS grid spacing                                      */
    int64_t src_sz[3];
    int64_t dst_sz[3];      /* affine: output dims; TPS: must equal src_sz           */
    double M[16];           /* affine matrix (kind 0)                                */
    const tw_marker *centres, *values; /* TPS landmarks (kind 1), copied at submit   */
    int n;
    double lambda;          /* 0 = 0.2                                               */
    const void *src;        /* input: host (pinned or pageable) memory, copied to HBM
                               after submit, or device memory, read in place         */
    void *dst;              /* output: host memory (copied back) or device memory
                               (written in place), complete when the job reports done */
} tw_job;

/* Continuous-batching server: a worker thread admits submitted jobs as soon
 * as the HBM budget allows, overlaps their transfers and kernels on a pool
 * of streams, and batches the resample work of all admitted jobs into one
 * persistent launch per round.  No counterpart in the reference. */
tw_status tw_server_create(tw_ctx *ctx, size_t hbm_budget_bytes, int max_inflight, tw_server **out);
tw_status tw_server_submit(tw_server *s, const tw_job *job, uint64_t *job_id);
/* TW_OK when done (latency_s = submit -> result in host memory),
 * TW_ERR_NOT_READY while running, or the job's error. */
tw_status tw_server_poll(tw_server *s, uint64_t job_id, double *latency_s);
tw_status tw_server_wait(tw_server *s, uint64_t job_id, double timeout_s, double *latency_s);
/* Stage times of a finished job, in seconds (-1 where a stage does not apply):
 *   times[0] submit -> admission (host clock: queued behind the HBM budget
 *            or the in-flight bound)
 *   times[1..6] from admission, on the GPU clock (CUDA events): solve done,
 *            node grid done, inputs resident, resample round started,
 *            resample round ended, result in place (copied back, or written
 *            in place for a device-resident job)
 *   times[7] submit -> done (host clock, the latency tw_server_poll reports)
 * TW_ERR_NOT_READY while the job runs.  No counterpart in the reference. */
tw_status tw_server_job_times(tw_server *s, uint64_t job_id, double times[8]);
tw_status tw_server_destroy(tw_server *s);

#ifdef __cplusplus
}
#endif

#endif /* TERAWARP_B200_H */
