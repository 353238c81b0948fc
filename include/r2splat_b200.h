/*
 * r2splat_b200 -- C ABI of the B200 (sm_100a) CT operator library.
 *
 * Every entry point takes raw device pointers, sizes, scalars, a dtype tag
 * (R2S_F32 / R2S_F64) and a cudaStream_t passed as void*. Entry points never
 * allocate device memory: outputs and scratch workspaces are supplied by the
 * caller (the Python shim allocates them through the torch caching
 * allocator). Work is enqueued on the given stream on the CURRENT device.
 * Each call returns R2S_OK (0) or an error code; r2s_last_error() returns a
 * thread-local message for the most recent failure.
 *
 * Each operator replaces one pybind11 binding of the reference
 * (MedAPT-group/R2Splat, r2splat/cuda/csrc/ext.cpp) whose C++ declaration is
 * cited as "Ops.h:line" (r2splat/cuda/include/Ops.h). Where the reference
 * binding allocates its outputs, the caller here passes them; where it returns
 * an undefined tensor (absgrad off), the corresponding pointer is NULL.
 * Array layouts are the reference's: contiguous row-major tensors.
 */
#ifndef R2SPLAT_B200_H
#define R2SPLAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define R2S_OK 0
#define R2S_ERR_ARGUMENT 1    /* invalid shape, size or pointer */
#define R2S_ERR_CUDA 2        /* a CUDA runtime call or kernel launch failed */
#define R2S_ERR_UNSUPPORTED 3 /* sizes beyond what this build supports */
#define R2S_ERR_WORKSPACE 4   /* workspace too small */

#define R2S_F32 0
#define R2S_F64 1

/* Library identification. */
int r2s_abi_version(void);
const char* r2s_last_error(void);

/* Measurement helper (no reference counterpart): launches blocks x threads
 * threads that each run iters x 128 independent FP32 FMAs, to measure the
 * FP32 issue peak the accumulate kernels are compared against. */
int r2s_fp32_peak_probe(float* out, uint32_t blocks, uint32_t threads, int iters, void* stream);

/* Measurement helper (no reference counterpart): blocks x threads threads
 * that each run iters x 128 independent fast base-2 exponentials (one SFU ex2
 * each), to measure the SFU issue peak of the exp/pow-bound loops. */
int r2s_sfu_peak_probe(float* out, uint32_t blocks, uint32_t threads, int iters, void* stream);

/* Number of kernels this library has launched in the process so far. */
uint64_t r2s_launch_count(void);

/* ------------------------------------------------------- input value checks
 * Batched form of the value checks of r2splat/_validation.py:35-48 (_tensor's
 * finiteness), :63-86 (_primitives' ranges) and r2splat/explicit.py's camera
 * checks: one launch evaluates up to 32 checks and sets bit `bit` of *flags
 * (cleared first) for each check that fails on any element, so the caller
 * reads one word instead of one host read per check. Elements are counted in
 * units of the check: scalars for FINITE / POSITIVE / NONNEGATIVE, rows of 4
 * for ZERO_ROW4, 3x3 matrices for FOCAL / PINHOLE, 4x4 for HOMOGENEOUS_ROW. */
#define R2S_CHECK_FINITE 0          /* fails on a non-finite value */
#define R2S_CHECK_ZERO_ROW4 1       /* fails on a row of four zeros (quaternion) */
#define R2S_CHECK_POSITIVE 2        /* fails on a value <= 0 */
#define R2S_CHECK_NONNEGATIVE 3     /* fails on a value < 0 */
#define R2S_CHECK_FOCAL 4           /* fails on K[0][0] <= 0 or K[1][1] <= 0 */
#define R2S_CHECK_PINHOLE 5         /* fails on nonzero skew or a last row other than [0, 0, 1] */
#define R2S_CHECK_HOMOGENEOUS_ROW 6 /* fails on a last row other than [0, 0, 0, 1] */
typedef struct {
    const void* data;
    uint64_t count;
    uint32_t kind;
    uint32_t bit;
} r2s_value_check;
int r2s_check_values(int dtype, const r2s_value_check* checks, uint32_t n_checks, uint32_t* flags,
                     void* stream);

/* ---------------------------------------------------------------- geometry */

/* Ops.h:419-422 parameter_transform_fwd_tensor.
 * quats [N,4] (wxyz, unnormalised), scales [N,3] -> covars [N,6], max_scales [N]. */
int r2s_parameter_transform_fwd(int dtype, const void* quats, const void* scales,
                                void* covars, void* max_scales, uint32_t n, void* stream);

/* Ops.h:424-428 parameter_transform_bwd_tensor. -> v_quats [N,4], v_scales [N,3]. */
int r2s_parameter_transform_bwd(int dtype, const void* quats, const void* scales,
                                const void* v_covars, void* v_quats, void* v_scales,
                                uint32_t n, void* stream);

/* Ops.h:397-406 world_to_image_projection_fwd_tensor.
 * means [N,3], covars [N,6], viewmats [C,4,4], Ks [C,3,3]
 * -> means2d [C,N,2], cov2d [C,N,6], radii [C,N,2] int32. */
int r2s_world_to_image_projection_fwd(int dtype, const void* means, const void* covars,
                                      const void* viewmats, const void* Ks, uint32_t C, uint32_t N,
                                      uint32_t width, uint32_t height, float eps_blur,
                                      float radius_clip, void* means2d, void* cov2d,
                                      int32_t* radii, void* stream);

/* Ops.h:408-417 world_to_image_projection_bwd_tensor. -> v_means [N,3], v_covars [N,6].
 * Sums over cameras per primitive in a fixed order (no atomics). */
int r2s_world_to_image_projection_bwd(int dtype, const void* means, const void* covars,
                                      const void* viewmats, const void* Ks, uint32_t C, uint32_t N,
                                      uint32_t width, uint32_t height, const void* v_means2d,
                                      const void* v_cov2d, void* v_means, void* v_covars,
                                      void* stream);

/* Ops.h:214-217 conics_mu_fwd_tensor. cov2d [total,6] -> conics [total,3], mus [total]. */
int r2s_conics_mu_fwd(int dtype, const void* cov2d, uint32_t total, double eps,
                      void* conics, void* mus, void* stream);

/* Ops.h:219-225 conics_mu_bwd_tensor. -> v_cov2d [total,6]. */
int r2s_conics_mu_bwd(int dtype, const void* cov2d, uint32_t total, double eps,
                      const void* conics, const void* mus, const void* v_conics,
                      const void* v_mus, void* v_cov2d, void* stream);

/* Ops.h:430-441 world_to_volume_mapping_fwd_tensor.
 * -> means3d_v [N,3], conics [N,6], radii [N,3] int32. (max_scales is unused, as in the reference.) */
int r2s_world_to_volume_mapping_fwd(int dtype, const void* means, const void* covars,
                                    const void* ranges, const void* centers, uint32_t N,
                                    uint32_t dim2, uint32_t dim1, uint32_t dim0, double eps3d,
                                    double radius_clip, void* means3d_v, void* conics,
                                    int32_t* radii, void* stream);

/* Ops.h:443-454 world_to_volume_mapping_bwd_tensor. -> v_means [N,3], v_covars [N,6]. */
int r2s_world_to_volume_mapping_bwd(int dtype, const void* means, const void* covars,
                                    const void* ranges, const void* centers, uint32_t N,
                                    uint32_t dim2, uint32_t dim1, uint32_t dim0, double eps3d,
                                    const void* v_means3d_v, const void* v_conics, void* v_means,
                                    void* v_covars, void* stream);

/* ------------------------------------------------- tile intersection (2D/3D)
 * Ops.h:46-52 isect_tiles_tensor, Ops.h:54-58 isect_offset_encode_tensor,
 * Ops.h:60-67 isect_tiles_3d_tensor, Ops.h:69-73 isect_offset_encode_3d_tensor.
 *
 * The reference's single call is split at the host read of the intersection
 * count (IsectTiles.cpp:95-100 reads it with .item()):
 *   1. r2s_isect_*_count: per-element tile counts (int32) and their inclusive
 *      prefix sum (int64). The caller reads cum_tiles[n_elems-1].
 *   2. r2s_isect_*_emit: writes the intersections sorted by key with ties in
 *      ascending element order (the order of the reference's stable radix
 *      sort), and optionally the per-key start offsets.
 * Keys: 2D = camera * tiles_x * tiles_y + tile_y * tiles_x + tile_x (element
 * c*N+n); 3D = (tz * tiles_y + ty) * tiles_x + tx (element n).
 * radii: 2D [C,N] (square) or [C,N,2] (rect, radii_is_rect=1); 3D [N,3].
 */
size_t r2s_isect_count_workspace(uint64_t n_elems);
size_t r2s_isect_emit_workspace(uint64_t n_isects, uint64_t n_keys);

int r2s_isect_tiles_count(int dtype, const void* means2d, const int32_t* radii, int radii_is_rect,
                          uint32_t C, uint32_t N, uint32_t tile_size, uint32_t tiles_x,
                          uint32_t tiles_y, int32_t* tiles_per_gauss, int64_t* cum_tiles,
                          void* workspace, size_t workspace_bytes, void* stream);
int r2s_isect_tiles_emit(int dtype, const void* means2d, const int32_t* radii, int radii_is_rect,
                         uint32_t C, uint32_t N, uint32_t tile_size, uint32_t tiles_x,
                         uint32_t tiles_y, const int64_t* cum_tiles, int64_t n_isects,
                         int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets,
                         void* workspace, size_t workspace_bytes, void* stream);
int r2s_isect_offset_encode(const int64_t* isect_ids, int64_t n_isects, uint32_t C,
                            uint32_t tiles_x, uint32_t tiles_y, int32_t* offsets, void* stream);

int r2s_isect_tiles_3d_count(int dtype, const void* means3d, const int32_t* radii, uint32_t N,
                             uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                             uint32_t tiles_z, int32_t* tiles_per_gauss, int64_t* cum_tiles,
                             void* workspace, size_t workspace_bytes, void* stream);
int r2s_isect_tiles_3d_emit(int dtype, const void* means3d, const int32_t* radii, uint32_t N,
                            uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                            uint32_t tiles_z, const int64_t* cum_tiles, int64_t n_isects,
                            int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets,
                            void* workspace, size_t workspace_bytes, void* stream);
int r2s_isect_offset_encode_3d(const int64_t* isect_ids, int64_t n_isects, uint32_t tiles_x,
                               uint32_t tiles_y, uint32_t tiles_z, int32_t* offsets, void* stream);

/* ------------------------------------------------------------ rasterization
 * Common arguments of the rasterize family (Ops.h:227-396):
 *   means2d [C,N,2], conics [C,N,3], opacities [C,N], mus [C,N],
 *   betas [C,N] (Beta variants; the projected exponent beta+1/2),
 *   uncertainties [N] (mean/variance variants), tile_offsets [C,ty,tx],
 *   flatten_ids [n_isects], isect_ids [n_isects] (per-primitive variants).
 *   width = dim1, height = dim0.
 * Workspace: r2s_raster_workspace(C, N, with_gradients) bytes.
 */
size_t r2s_raster_workspace(uint32_t dtype, uint32_t C, uint32_t N, int with_gradients);

/* Ops.h:227-236 rasterize_to_pixels_fwd_tensor / Ops.h:309-319 beta_rasterize_to_pixels_fwd_tensor
 * (betas NULL selects the Gaussian kernel). -> render [C,H,W]. */
int r2s_rasterize_to_pixels_fwd(int dtype, const void* means2d, const void* conics,
                                const void* opacities, const void* mus, const void* betas,
                                const int32_t* tile_offsets, const int32_t* flatten_ids,
                                uint32_t C, uint32_t N, uint32_t n_isects, uint32_t width,
                                uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, void* render, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Ops.h:238-248 rasterize_to_pixels_mean_var_fwd_tensor / Ops.h:321-332 beta_... -> render, render_var. */
int r2s_rasterize_to_pixels_mean_var_fwd(int dtype, const void* means2d, const void* conics,
                                         const void* opacities, const void* mus, const void* betas,
                                         const void* uncertainties, const int32_t* tile_offsets,
                                         const int32_t* flatten_ids, uint32_t C, uint32_t N,
                                         uint32_t n_isects, uint32_t width, uint32_t height,
                                         uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                                         void* render, void* render_var, void* workspace,
                                         size_t workspace_bytes, void* stream);

/* Ops.h:250-260 rasterize_to_pixels_uncertainty_bwd_tensor / Ops.h:334-345 beta_...
 * -> v_uncertainties [N] (zeroed by the call). */
int r2s_rasterize_to_pixels_uncertainty_bwd(int dtype, const void* means2d, const void* conics,
                                            const void* opacities, const void* mus,
                                            const void* betas, const int32_t* tile_offsets,
                                            const int32_t* flatten_ids, const void* v_render_var,
                                            uint32_t C, uint32_t N, uint32_t n_isects,
                                            uint32_t width, uint32_t height, uint32_t tile_size,
                                            uint32_t tiles_x, uint32_t tiles_y,
                                            void* v_uncertainties, void* workspace,
                                            size_t workspace_bytes, void* stream);

/* Ops.h:262-274 rasterize_to_pixels_bwd_tensor ("pixel" mode),
 * Ops.h:276-289 rasterize_to_pixels_bwd_per_gaussian_tensor ("primitive" mode),
 * Ops.h:291-307 rasterize_to_pixels_mean_var_bwd_per_gaussian_tensor, and the
 * Beta counterparts Ops.h:347-396. One entry point serves all of them:
 *   betas NULL -> Gaussian; v_render_var NULL -> plain VJP;
 *   uncertainties NULL with v_render_var set -> detached variance branch
 *   (ext.cpp:106-128 overload); v_means2d_abs NULL -> absgrad off;
 *   v_betas required iff betas; v_uncertainties required iff v_render_var.
 * isect_ids may be NULL (the tile of each intersection is implied by the
 * offsets). Outputs (all zeroed by the call): v_means2d [C,N,2],
 * v_conics [C,N,3], v_opacities [C,N], v_mus [C,N], v_betas [C,N],
 * v_uncertainties [N], v_means2d_abs [C,N,2]. */
int r2s_rasterize_to_pixels_bwd(int dtype, const void* means2d, const void* conics,
                                const void* opacities, const void* mus, const void* betas,
                                const int32_t* tile_offsets, const int64_t* isect_ids,
                                const int32_t* flatten_ids, const void* v_render,
                                const void* v_render_var, const void* uncertainties,
                                uint32_t C, uint32_t N, uint32_t n_isects, uint32_t width,
                                uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, void* v_means2d_abs, void* v_means2d,
                                void* v_conics, void* v_opacities, void* v_mus, void* v_betas,
                                void* v_uncertainties, void* workspace, size_t workspace_bytes,
                                void* stream);

/* ---------------------------------------------------------- voxelization
 * Common arguments (Ops.h:75-212): means3d [N,3], conics [N,6],
 * opacities [N], betas [N] (Beta), uncertainties [N] (mean/variance),
 * tile_offsets [tz,ty,tx], flatten_ids [n_isects]; dim2 = x, dim1 = y, dim0 = z.
 * Workspace: r2s_voxel_workspace(N, with_gradients) bytes.
 */
size_t r2s_voxel_workspace(uint32_t dtype, uint32_t N, int with_gradients);

/* Ops.h:75-84 voxelize_to_voxels_fwd_tensor / Ops.h:142-152 beta_... -> volume [D,H,W]. */
int r2s_voxelize_to_voxels_fwd(int dtype, const void* means3d, const void* conics,
                               const void* opacities, const void* betas,
                               const int32_t* tile_offsets, const int32_t* flatten_ids,
                               uint32_t N, uint32_t n_isects, uint32_t dim2, uint32_t dim1,
                               uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                               uint32_t tiles_y, uint32_t tiles_z, void* volume, void* workspace,
                               size_t workspace_bytes, void* stream);

/* Ops.h:86-96 voxelize_to_voxels_mean_var_fwd_tensor / Ops.h:154-165 beta_... */
int r2s_voxelize_to_voxels_mean_var_fwd(int dtype, const void* means3d, const void* conics,
                                        const void* opacities, const void* betas,
                                        const void* uncertainties, const int32_t* tile_offsets,
                                        const int32_t* flatten_ids, uint32_t N, uint32_t n_isects,
                                        uint32_t dim2, uint32_t dim1, uint32_t dim0,
                                        uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                                        uint32_t tiles_z, void* volume, void* volume_var,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* Ops.h:98-140 voxelize_to_voxels_bwd / _bwd_per_gaussian / _mean_var_bwd_per_gaussian
 * and the Beta counterparts Ops.h:167-212 (ext.cpp:42-94 overloads). Same NULL
 * conventions as r2s_rasterize_to_pixels_bwd. Outputs (zeroed by the call):
 * v_means3d [N,3], v_conics [N,6], v_opacities [N], v_betas [N], v_uncertainties [N]. */
int r2s_voxelize_to_voxels_bwd(int dtype, const void* means3d, const void* conics,
                               const void* opacities, const void* betas,
                               const int32_t* tile_offsets, const int64_t* isect_ids,
                               const int32_t* flatten_ids, const void* v_volume,
                               const void* v_volume_var, const void* uncertainties, uint32_t N,
                               uint32_t n_isects, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                               uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t tiles_z, void* v_means3d, void* v_conics,
                               void* v_opacities, void* v_betas, void* v_uncertainties,
                               void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ losses */

/* Ops.h:37-39 volume_loss_fwd (anisotropic TV over [B,D,H,W]).
 * -> loss [1], tv [1], tv_map [B,D,H,W] (tv_map may be NULL to skip writing it).
 * Workspace: r2s_volume_loss_workspace(numel). */
size_t r2s_volume_loss_workspace(uint64_t numel);
int r2s_volume_loss_fwd(int dtype, const void* volume, uint32_t B, uint32_t D, uint32_t H,
                        uint32_t W, float lambda_tv, void* loss, void* tv, void* tv_map,
                        void* workspace, size_t workspace_bytes, void* stream);
/* Ops.h:41-44 volume_loss_bwd. grad_output [1] -> grad_volume [B,D,H,W] (lambda folded in). */
int r2s_volume_loss_bwd(int dtype, const void* volume, const void* grad_output, uint32_t B,
                        uint32_t D, uint32_t H, uint32_t W, float lambda_tv, void* grad_volume,
                        void* stream);

/* Ops.h:37-44 volume_loss_fwd followed by volume_loss_bwd, as one pass over the volume, for
 * callers that know the upstream gradient grad_output [1] (device) before the forward, as a fit
 * step does. -> loss [1], tv [1], tv_map [B,D,H,W] (optional, null to skip), grad_volume
 * [B,D,H,W]. tv_map and grad_volume equal the two calls' bit for bit. Workspace:
 * r2s_volume_loss_workspace(numel). */
int r2s_volume_loss_fwd_bwd(int dtype, const void* volume, const void* grad_output, uint32_t B,
                            uint32_t D, uint32_t H, uint32_t W, float lambda_tv, void* loss,
                            void* tv, void* tv_map, void* grad_volume, void* workspace,
                            size_t workspace_bytes, void* stream);

/* Ops.h:15-18 image_loss_fwd / Ops.h:26-29 image_loss_l1_fwd (mean L1 over [B,H,W]).
 * -> loss [1], l1 [1], l1_map [B,H,W]. Workspace: r2s_volume_loss_workspace(numel). */
int r2s_image_loss_l1_fwd(int dtype, const void* prediction, const void* target, uint32_t B,
                          uint32_t H, uint32_t W, float lambda_l1, void* loss, void* l1,
                          void* l1_map, void* workspace, size_t workspace_bytes, void* stream);
/* Ops.h:20-24 image_loss_bwd / Ops.h:31-35 image_loss_l1_bwd. -> grad_prediction [B,H,W]. */
int r2s_image_loss_l1_bwd(int dtype, const void* prediction, const void* target,
                          const void* grad_output, uint32_t B, uint32_t H, uint32_t W,
                          float lambda_l1, void* grad_prediction, void* stream);

/* ------------------------------------------- fused explicit-operator path
 * These have no single reference counterpart: they implement the pipelines of
 * the reference's r2splat/explicit.py (rasterize_fwd :102-188,
 * rasterize_bwd :191-242, voxelize_fwd :245-311, voxelize_bwd :314-351) with
 * fewer passes over HBM.
 */

/* Projection + conic/mu + packing (explicit.py:160-170). Writes one 8-slot
 * record per (camera, primitive) -- x, y, a, b, c, density, mu, beta+1/2 --
 * into records [C,N,8], the tile rectangle rects [C,N,4] (uint16: x0, y0, x1, y1),
 * and tiles_per_gauss [C,N]. ratio [N] (Beta path factor) and betas [N] may
 * be NULL for Gaussians. */
int r2s_raster_project(int dtype, const void* means, const void* covars, const void* densities,
                       const void* betas, const void* ratio, const void* viewmats, const void* Ks,
                       uint32_t C, uint32_t N, uint32_t width, uint32_t height, float eps_blur,
                       double eps, float radius_clip, uint32_t tile_size, uint32_t tiles_x,
                       uint32_t tiles_y, void* records, uint16_t* rects, int32_t* tiles_per_gauss,
                       void* stream);

/* Inclusive prefix sum of int32 tile counts into int64 (the reference's
 * torch::cumsum(..., kInt64), IsectTiles.cpp:95-97). Workspace: r2s_isect_count_workspace(n). */
int r2s_scan_tile_counts(const int32_t* counts, uint64_t n, int64_t* cum, void* workspace,
                         size_t workspace_bytes, void* stream);

/* Emits the sorted 2D intersections from precomputed rectangles (no radii). */
int r2s_raster_emit(const uint16_t* rects, uint32_t C, uint32_t N, uint32_t tiles_x,
                    uint32_t tiles_y, const int64_t* cum_tiles, int64_t n_isects,
                    int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets, void* workspace,
                    size_t workspace_bytes, void* stream);

/* Tile accumulation on packed records. uncertainties [N] for the variance image. */
int r2s_raster_render(int dtype, const void* records, const void* uncertainties, int beta,
                      const int32_t* tile_offsets, const int32_t* flatten_ids, uint32_t C,
                      uint32_t N, uint32_t n_isects, uint32_t width, uint32_t height,
                      uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, void* render,
                      void* render_var, void* stream);

/* Tile VJP on packed records, accumulating packed per-(camera, primitive)
 * adjoints grads [C,N,8] (x, y, a, b, c, density, mu, beta) and
 * v_uncertainties [N]; both must be zeroed by the caller. */
int r2s_raster_render_bwd(int dtype, const void* records, const void* uncertainties, int beta,
                          int detach_variance, const int32_t* tile_offsets,
                          const int32_t* flatten_ids, const void* v_render,
                          const void* v_render_var, uint32_t C, uint32_t N, uint32_t n_isects,
                          uint32_t width, uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                          uint32_t tiles_y, void* grads, void* v_means2d_abs,
                          void* v_uncertainties, void* stream);

/* Record-parallel VJP of r2s_raster_render: one pass over the [C,N] records
 * (not the intersection lists), each record evaluated on the pixels of its
 * tile rectangle rects [C,N,4] (uint16 x0, y0, x1, y1 in tiles, upper bounds
 * exclusive, as r2s_raster_project writes them) and written to grads [C,N,8]
 * without atomics (every record written; the buffer needs no clearing).
 * v_means2d_abs [C,N,2] optional (written); v_uncertainties [C,N] with the
 * variance branch: each record's uncertainty adjoint (written), to be summed
 * over cameras by r2s_sum_over_cameras, so the result does not depend on the
 * order the records finish in. Same adjoints as r2s_raster_render_bwd. */
int r2s_raster_record_bwd(int dtype, const void* records, const uint16_t* rects, const void* uncertainties,
                          int beta, int detach_variance, const void* v_render, const void* v_render_var,
                          uint32_t C, uint32_t N, uint32_t width, uint32_t height, uint32_t tile_size,
                          void* grads, void* v_means2d_abs, void* v_uncertainties, void* stream);

/* out [N] = sum over cameras c of per_record [C,N], in camera order (the
 * record VJP's uncertainty adjoints; no reference counterpart as a call: the
 * reference adds them with atomics inside K20/K22). */
int r2s_sum_over_cameras(int dtype, const void* per_record, uint32_t C, uint32_t N, void* out, void* stream);

/* Chain rule from packed adjoints to physical parameters (explicit.py:225-241):
 * conic/mu VJP, projection VJP summed over cameras, Beta path factor and the
 * parameter-transform VJP, per primitive, with no atomics. log_grad [N] and
 * ratio [N] only for Beta. -> v_means [N,3], v_quats [N,4], v_scales [N,3],
 * v_densities [N], v_betas [N] (Beta). */
int r2s_raster_chain_bwd(int dtype, const void* means, const void* quats, const void* scales,
                         const void* covars, const void* betas, const void* ratio,
                         const void* log_grad, const void* viewmats, const void* Ks, uint32_t C,
                         uint32_t N, uint32_t width, uint32_t height, float eps_blur, double eps,
                         const void* grads, void* v_means, void* v_quats, void* v_scales,
                         void* v_densities, void* v_betas, void* stream);

/* Volume mapping + packing (explicit.py:290-294): records [N,16] (x, y, z, density,
 * six conic entries, beta, uncertainty, padding), voxel-space means means_v [N,3],
 * radii [N,3], tiles_per_gauss [N]. */
int r2s_voxel_project(int dtype, const void* means, const void* covars, const void* densities,
                      const void* betas, const void* uncertainties, const void* ranges,
                      const void* centers, uint32_t N, uint32_t dim2, uint32_t dim1,
                      uint32_t dim0, double eps3d, double radius_clip, uint32_t tile_size,
                      uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, void* records,
                      void* means_v, int32_t* radii, int32_t* tiles_per_gauss, void* stream);

int r2s_voxel_render(int dtype, const void* records, int beta, const int32_t* tile_offsets,
                     const int32_t* flatten_ids, uint32_t N, uint32_t n_isects, uint32_t dim2,
                     uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                     uint32_t tiles_y, uint32_t tiles_z, void* volume, void* volume_var,
                     void* stream);

/* Voxel tile VJP into packed adjoints grads [N,16] (x, y, z, density, six conic
 * entries, beta, uncertainty, ...), zeroed by the caller. */
int r2s_voxel_render_bwd(int dtype, const void* records, int beta, int detach_variance,
                         const int32_t* tile_offsets, const int32_t* flatten_ids,
                         const void* v_volume, const void* v_volume_var, uint32_t N,
                         uint32_t n_isects, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                         uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z,
                         void* grads, void* stream);

/* Chain rule for voxelization (explicit.py:343-351). */
int r2s_voxel_chain_bwd(int dtype, const void* means, const void* quats, const void* scales,
                        const void* covars, const void* ranges, const void* centers, uint32_t N,
                        uint32_t dim2, uint32_t dim1, uint32_t dim0, double eps3d,
                        const void* grads, void* v_means, void* v_quats, void* v_scales,
                        void* v_densities, void* v_betas, void* v_uncertainties, void* stream);

/* ------------------------------------------- capacity-bounded (graph) mode
 * No reference counterpart: variants of the fused pipeline whose intersection
 * count stays on the device, so a whole fit step can be captured in a CUDA
 * graph (no host read of the count). The lists live in buffers of a fixed
 * `capacity`; *n_used receives the count (0 when it exceeds the capacity, in
 * which case nothing is written past the capacity and *overflow gets bit 0
 * set; the caller clears *overflow, grows the capacity and repeats the step).
 * Workspace: r2s_isect_emit_workspace(capacity, n_keys). The render entries
 * read the count from n_used. */
int r2s_raster_emit_capacity(const uint16_t* rects, uint32_t C, uint32_t N, uint32_t tiles_x, uint32_t tiles_y,
                             const int64_t* cum_tiles, int64_t capacity, int64_t* n_used, uint32_t* overflow,
                             int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets, void* workspace,
                             size_t workspace_bytes, void* stream);
int r2s_voxel_emit_capacity(int dtype, const void* means3d, const int32_t* radii, uint32_t N, uint32_t tile_size,
                            uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, const int64_t* cum_tiles,
                            int64_t capacity, int64_t* n_used, uint32_t* overflow, int64_t* isect_ids,
                            int32_t* flatten_ids, int32_t* offsets, void* workspace, size_t workspace_bytes,
                            void* stream);
/* stage_batch: records staged in shared memory per batch of the tile kernel
 * (0 = the default 256; capped at the kernel's thread count). */
int r2s_raster_render_capacity(int dtype, const void* records, const void* uncertainties, int beta,
                               const int32_t* tile_offsets, const int32_t* flatten_ids, const int64_t* n_used,
                               uint32_t C, uint32_t N, uint32_t width, uint32_t height, uint32_t tile_size,
                               uint32_t tiles_x, uint32_t tiles_y, uint32_t stage_batch, void* render,
                               void* render_var, void* stream);
int r2s_voxel_render_capacity(int dtype, const void* records, int beta, const int32_t* tile_offsets,
                              const int32_t* flatten_ids, const int64_t* n_used, uint32_t N, uint32_t dim2,
                              uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                              uint32_t tiles_z, void* volume, void* volume_var, void* stream);
int r2s_voxel_render_bwd_capacity(int dtype, const void* records, int beta, int detach_variance,
                                  const int32_t* tile_offsets, const int32_t* flatten_ids, const int64_t* n_used,
                                  const void* v_volume, const void* v_volume_var, uint32_t N, uint32_t dim2,
                                  uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                                  uint32_t tiles_y, uint32_t tiles_z, void* grads, void* stream);

/* Deterministic form of r2s_voxel_render_bwd (the explicit path's voxel VJP; the
 * reference's K30/K32, VoxelizeToVoxelsBwd.cu:322-514, add every (tile, primitive)
 * pair's sums into the primitive's adjoints with atomics). Each pair writes its 12
 * sums to slot tile_cum[n - 1] + (the tile's index in primitive n's 3D tile box,
 * z then y then x), and a second pass adds each primitive's slots in a fixed order into
 * grads [N] (written, not accumulated): the same result on every run. means_v [N,3]
 * and radii [N,3] are r2s_voxel_project's (the tile box is taken from the records'
 * voxel-space centre, which r2s_voxel_project writes equal to means_v), tile_cum [N]
 * int64 the inclusive scan of its tile counts; slots [slot_capacity, 12] is caller
 * scratch, 16-byte aligned, slot_capacity below 2^31. Capacity-bounded form: n_used (device count)
 * instead of n_isects; slots past slot_capacity are neither written nor read (such a
 * step overflowed and is discarded). */
int r2s_voxel_render_bwd_slots(int dtype, const void* records, int beta, int detach_variance,
                               const int32_t* tile_offsets, const int32_t* flatten_ids, uint64_t n_isects,
                               const int64_t* n_used, const void* means_v, const int32_t* radii,
                               const int64_t* tile_cum, const void* v_volume, const void* v_volume_var, uint32_t N,
                               uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                               uint32_t tiles_y, uint32_t tiles_z, void* slots, uint64_t slot_capacity, void* grads,
                               void* stream);

/* Per-tile packed record layout of the 3D tile pipeline (replaces the reference's
 * per-intersection gathers through flatten_ids in K29-K32, VoxelizeToVoxelsFwd.cu:73-139
 * and VoxelizeToVoxelsBwd.cu:322-380, which read means3d/conics/opacities at
 * g = flatten_ids[i] for every list entry). packed [n_isects] Rec3D (64 B fp32,
 * 128 B fp64, caller-allocated) receives records[flatten_ids[i]] for each sorted
 * intersection i, so a tile's list is one contiguous range that the tile kernels stage
 * with one bulk copy per batch. The padding carries the pair's VJP slot, as in
 * r2s_voxel_render_bwd_slots (0xffffffff past slot_capacity). tile_offsets and
 * flatten_ids are the sorted 3D lists, radii [N,3] and tile_cum [N] r2s_voxel_project's
 * and its tile-count scan; workspace holds r2s_voxel_pack_workspace(N) bytes.
 * Capacity-bounded form: n_isects is the capacity and n_used the device count. */
size_t r2s_voxel_pack_workspace(uint32_t N);
int r2s_voxel_pack_tile_records(int dtype, const void* records, const int32_t* tile_offsets,
                                const int32_t* flatten_ids, const int32_t* radii, const int64_t* tile_cum, uint32_t N,
                                uint64_t n_isects, const int64_t* n_used, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, uint32_t tiles_z, uint64_t slot_capacity, void* packed,
                                void* workspace, size_t workspace_bytes, void* stream);
/* r2s_voxel_render (K29/K31) on the packed layout: the same volume and variance bit for
 * bit. n_used null: n_isects is the count; else the device count (n_isects unused). */
int r2s_voxel_render_packed(int dtype, const void* packed, int beta, const int32_t* tile_offsets,
                            uint64_t n_isects, const int64_t* n_used, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                            uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, void* volume,
                            void* volume_var, void* stream);
/* r2s_voxel_render_bwd_slots (K30/K32, deterministic slots) on the packed layout, with
 * the slots taken from the records' padding: the same grads bit for bit. */
int r2s_voxel_render_bwd_packed(int dtype, const void* packed, int beta, int detach_variance,
                                const int32_t* tile_offsets, uint64_t n_isects, const int64_t* n_used,
                                const int64_t* tile_cum, const void* v_volume, const void* v_volume_var, uint32_t N,
                                uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, uint32_t tiles_z, void* slots, uint64_t slot_capacity, void* grads,
                                void* stream);
/* Number of bulk-staging waits on `device` that ran out (a batch copy that did not
 * complete within 0.2 s; the kernel then left the rest of that tile unwritten) since
 * the last clear; clear != 0 resets it. Synchronous: reads a device word. No
 * counterpart in the reference (its tile kernels stage with plain loads). */
int r2s_bulk_wait_faults(int device, int clear, uint32_t* count);

/* Record-parallel voxel VJP, for a backward that keeps no intersection lists
 * (recompute-in-backward under a memory budget), replacing the tile-parallel
 * per-primitive VJP with atomics (VoxelizeToVoxelsBwd.cu:322-514, K30/K32, for
 * the path explicit.py:331-350 drives). A work item is one primitive and one
 * z-layer of its 3D tile box (IsectTiles3DKernel.cu:38-112); it needs no sorted
 * lists. r2s_voxel_layer_counts writes each primitive's layer count [N] int32
 * from the voxel-space means and radii of r2s_voxel_project; its inclusive
 * scan (r2s_scan_tile_counts) is layer_cum [N] int64 and its total n_items.
 * r2s_voxel_record_bwd walks every item into partials [n_items] (64-byte
 * records) and sums each primitive's slots in layer order into grads [N]
 * (packed as r2s_voxel_render_bwd's, written, not accumulated): deterministic.
 * Capacity-bounded form: n_items is the capacity of partials and n_items_dev
 * the device-side total (layer_cum's last entry); a total above the capacity
 * sets *overflow (may be null) and the result is to be discarded. */
int r2s_voxel_layer_counts(int dtype, const void* means_v, const int32_t* radii, uint32_t N, uint32_t dim2,
                           uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                           uint32_t tiles_z, int32_t* layers, void* stream);
int r2s_voxel_record_bwd(int dtype, const void* records, const void* means_v, const int32_t* radii,
                         const int64_t* layer_cum, uint64_t n_items, const int64_t* n_items_dev, int beta,
                         int detach_variance, const void* v_volume, const void* v_volume_var, uint32_t N,
                         uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                         uint32_t tiles_y, uint32_t tiles_z, void* partials, void* grads, uint32_t* overflow,
                         void* stream);

/* ------------------------------------------ forward with fused image loss
 * Replaces, in a fit step, the separate image-loss pass after
 * rasterize_to_pixels_fwd (caller-side in examples/optimize.py; the L1 form is
 * image_loss_l1_fwd/bwd, Loss.cpp:12-113, ImageLossFwd.cu:19-31,
 * ImageLossBwd.cu:14-30). r2s_raster_render plus an epilogue: each pixel also
 * writes v_render = d(loss)/d(render) for the mean loss over the C*H*W pixels
 * and adds its term to a per-tile fp64 partial, summed in a fixed order:
 *   R2S_IMAGE_LOSS_MSE: loss = lambda * mean((render - target)^2),
 *                       v_render = (render - target) * (2 lambda / numel);
 *   R2S_IMAGE_LOSS_L1:  loss = lambda * mean|render - target|,
 *                       v_render = lambda * sign(render - target) / numel
 *                       (image_loss_l1_bwd with grad_output = 1).
 * loss_value = the mean without lambda. n_used, when non-NULL, overrides
 * n_isects (capacity-bounded mode). Workspace:
 * r2s_raster_image_loss_workspace(C, tiles_x, tiles_y). render must not
 * alias target or v_render. */
#define R2S_IMAGE_LOSS_MSE 0
#define R2S_IMAGE_LOSS_L1 1
size_t r2s_raster_image_loss_workspace(uint32_t C, uint32_t tiles_x, uint32_t tiles_y);
int r2s_raster_render_image_loss(int dtype, const void* records, const void* uncertainties, int beta,
                                 const int32_t* tile_offsets, const int32_t* flatten_ids, uint32_t n_isects,
                                 const int64_t* n_used, uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                 uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t stage_batch,
                                 const void* target, int loss_kind, float lambda, void* render, void* render_var,
                                 void* v_render, void* loss, void* loss_value, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* Fused fit-loop update, no reference counterpart (the reference's example
 * loop, examples/optimize.py, does it with torch ops): sums two physical VJPs
 * grads_a/grads_b (each an array of 5 pointers: means [N,3], quats [N,4],
 * scales [N,3], densities [N], beta [N] or NULL; grads_b may be NULL),
 * applies the activation derivatives of scales = exp(raw_scales), densities =
 * softplus(raw_densities), beta = exp(raw_beta), takes one Adam step (torch's
 * order of operations; moments [N,12]) on the raw parameters in place, writes
 * the activated scales/densities/beta, and advances *step. A nonzero *skip
 * makes the call a no-op. raw_beta and beta are both NULL without Beta. */
int r2s_adam_activation_step(int dtype, uint32_t N, void* means, void* quats, void* raw_scales, void* raw_densities,
                             void* raw_beta, void* scales, void* densities, void* beta, void* adam_m, void* adam_v,
                             const void* const* grads_a, const void* const* grads_b, double lr, double beta1,
                             double beta2, double eps, int32_t* step, const uint32_t* skip, void* stream);

/* ------------------------------------------------ allocation-free variant
 * No reference counterpart. r2s_scan_tile_counts without a workspace argument:
 * the scan's scratch is a static per-device array of the library (72 KiB),
 * so the call needs no device allocation at all. It takes at most
 * r2s_scan_tile_counts_noalloc_max() elements (2^25); larger n returns
 * R2S_ERR_UNSUPPORTED with nothing launched. Calls on one device share the
 * scratch: calls that overlap in time race and must be serialised by the
 * caller. The first call on a device resolves the scratch address and should
 * come before any stream capture on that device. The address stays cached for
 * the process, so a device must not be reset (cudaDeviceReset) after this
 * entry point has been called on it. */
uint64_t r2s_scan_tile_counts_noalloc_max(void);
int r2s_scan_tile_counts_noalloc(const int32_t* counts, uint64_t n, int64_t* cum, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* R2SPLAT_B200_H */
