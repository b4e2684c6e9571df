/*
 * jaxpower_b200: C ABI of the B200 (sm_100a) mesh power-spectrum kernels.
 *
 * Drop-in boundary for jax-power's single-GPU power-spectrum path.  Each entry
 * point replaces one reference function (cited below as path:line inside the
 * adematti/jax-power project).  All calls:
 *   - take plain device pointers and sizes, borrowed from the caller;
 *   - are ordered on the given CUDA stream (cudaStream_t passed as void*),
 *     with no hidden device synchronisation (except where stated);
 *   - take caller-owned workspace sized by the matching *_workspace_size();
 *   - return a pk_status; on error pk_last_error() describes it (thread local).
 *
 * Layouts: positions (n, 3) float32 row-major; weights (n,) float32 (NULL = 1);
 * real mesh (N0, N1, N2) float32 C order; complex mesh (N0, N1, N2/2+1)
 * interleaved complex64 (float2) C order (cuFFT R2C layout, the reference's
 * Hermitian layout of fft_backend='jax').
 */
#ifndef JAXPOWER_B200_H
#define JAXPOWER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int pk_status;
enum {
  PK_OK = 0,
  PK_ERR_INVALID = 1,   /* bad argument (sizes, orders, null pointers) */
  PK_ERR_CUDA = 2,      /* a CUDA runtime / cuFFT call failed */
  PK_ERR_WORKSPACE = 3, /* workspace too small */
  PK_ERR_RANGE = 4      /* input outside the supported range */
};

/* Fourier-layout semantics of the reference's two FFT backends
 * (mesh.py:1488-1489, 1679-1719): 0 = 'jax' (rfftn, Hermitian weights
 * 1 + (kz > 0)); 1 = 'jaxdecomp' (full complex FFT), reproduced on the
 * Hermitian storage (interlacing phase symmetrised, Nyquist-plane weight 1). */
enum { PK_BACKEND_JAX = 0, PK_BACKEND_JAXDECOMP = 1 };

const char *pk_version(void);
const char *pk_last_error(void);

/* ------------------------------------------------------------------ paint
 * Replaces resamplers.paint (resamplers.py:66-97) as driven by _paint
 * (mesh.py:2673-2729): positions are normalised as
 * (pos + boxsize/2 - boxcenter) / cellsize in float32 (mesh.py:2684), shifted
 * by shift_s = s / interlacing (mesh.py:2679) for s in
 * [shift_begin, shift_begin + nshifts) (nshifts <= 4) and painted with the
 * order-`order` B-spline (1 ngp, 2 cic, 3 tsc, 4 pcs) on the periodic mesh.
 * Writes nshifts real meshes, out[j * N0*N1*N2 + ...].  Deterministic: per-cell
 * sums are accumulated in 64-bit fixed point, independent of particle order.
 * cellsize[3] is boxsize / meshsize in float32 (mesh.py:1575).
 * d_status (device int, may be NULL) is set to 1 if a position or weight is
 * not finite or a position is more than 2^22 cells away; such particles are
 * skipped. */
pk_status pk_paint_workspace_size(int64_t n, const int32_t meshsize[3], int order,
                                  int nshifts, size_t *bytes);
pk_status pk_paint(void *stream, const float *positions, const float *weights, int64_t n,
                   const int32_t meshsize[3], const float boxsize[3],
                   const float boxcenter[3], const float cellsize[3], int order,
                   int interlacing, int shift_begin, int nshifts, float *out,
                   void *workspace, size_t workspace_bytes, int *d_status);

/* Batched paint of nmocks catalogs on the same mesh geometry in one set of launches:
 * positions / weights are concatenated, d_offsets (device, int64, nmocks + 1) gives
 * each catalog's range; out[(m * nshifts + j) * N0*N1*N2 + ...].  tile_config
 * (0..7) selects the tile shape / CTA size (0: 8x16x32 cells, 512 threads; 1: 8x16x32,
 * 256; 2: 8x8x32, 256; 3: 4x16x32, 256; 4..7: the same with shared-memory rows swizzled
 * against bank conflicts), for an autotuner; every configuration paints the same bits.
 * pk_paint is the nmocks = 1, tile_config = 4 case. */
pk_status pk_paint_batch_workspace_size(int64_t n, int nmocks, const int32_t meshsize[3],
                                        int order, int nshifts, int tile_config, size_t *bytes);
pk_status pk_paint_batch(void *stream, const float *positions, const float *weights,
                         const int64_t *d_offsets, int64_t n, int nmocks,
                         const int32_t meshsize[3], const float boxsize[3],
                         const float boxcenter[3], const float cellsize[3], int order,
                         int interlacing, int shift_begin, int nshifts, int tile_config,
                         float *out, void *workspace, size_t workspace_bytes, int *d_status);

/* Replaces resamplers.read (resamplers.py:100-125) via _read (mesh.py:2064-2110):
 * out[p] = sum_offsets mesh[wrap(i0 + off)] * W(u), u normalised as above plus
 * `shift`.  If grad (n, 3) is non-NULL, also writes
 * grad[p, d] = scale * w_p * sum_offsets mesh * dW/du_d / cellsize_d
 * (the position gradient of paint's adjoint); accumulate != 0 adds into
 * out / grad instead of overwriting. */
pk_status pk_read(void *stream, const float *mesh, const float *positions,
                  const float *weights, int64_t n, const int32_t meshsize[3],
                  const float boxsize[3], const float boxcenter[3], const float cellsize[3],
                  int order, float shift, float scale, float *out, float *grad,
                  int accumulate);

/* pk_read over the `interlacing` shifted meshes of an interlaced paint, mesh s at
 * meshes + s * N0 N1 N2 read at u + s / interlacing (the transpose of the shifted
 * paints of _paint, mesh.py:2737-2752): out[p] and grad[p] are the sums over s, added
 * in shift order, of what pk_read gives for each mesh (bit for bit the same as one
 * accumulating pk_read per shift). */
pk_status pk_read_interlaced(void *stream, const float *meshes, int interlacing,
                             const float *positions, const float *weights, int64_t n,
                             const int32_t meshsize[3], const float boxsize[3],
                             const float boxcenter[3], const float cellsize[3], int order,
                             float scale, float *out, float *grad, int accumulate);

/* ------------------------------------------------------------------- FFT
 * cuFFT plans for the reference's r2c / c2r (mesh.py:1679-1719): batch meshes
 * of shape meshsize, contiguous, out of place.  Both directions are
 * unnormalised; jnp.fft.irfftn's 1 / (N0 N1 N2) is folded by the caller into
 * the preceding pass (pk_interlace_compensate's scale) or pk_scale_real.
 * A C2R overwrites its input.  direction: 0 = R2C, 1 = C2R. */
typedef struct pk_fft_plan_s *pk_fft_plan;
pk_status pk_fft_plan_create(const int32_t meshsize[3], int batch, int direction,
                             pk_fft_plan *plan);
pk_status pk_fft_exec(pk_fft_plan plan, void *stream, void *in, void *out);
pk_status pk_fft_plan_destroy(pk_fft_plan plan);

/* ------------------------------------------- interlacing + compensation
 * Fused replacement of the interlacing accumulation (mesh.py:2737-2749),
 * compensation (resamplers.py:16-26, mesh.py:2733-2751) in one pass:
 *   out(k) = C(k) / I * sum_s in_s(k) * exp(i shift_s (kx_c + ky_c + kz_c))
 * with circular k (mesh.py:1627-1629), C = prod_d sinc(k_d/2pi)^-comp_order
 * (comp_order = 0: none).  for_c2r != 0 Hermitian-symmetrises the kz = 0 and
 * kz = N/2 planes so any C2R gives numpy's irfftn of the same data.
 * backend selects the 'jax' / 'jaxdecomp' semantics; the output is multiplied
 * by scale.  in holds the nshifts = interlacing shifted meshes (shift s / I);
 * in may equal out only when nshifts == 1 and for_c2r == 0. */
pk_status pk_interlace_compensate(void *stream, const void *in, int nshifts,
                                  const int32_t meshsize[3], int comp_order, int backend,
                                  int for_c2r, float scale, void *out);

/* The same for nbatch independent sets of nshifts meshes (in: nbatch * nshifts meshes,
 * out: nbatch meshes), in one launch. */
pk_status pk_interlace_compensate_batch(void *stream, const void *in, int nbatch, int nshifts,
                                        const int32_t meshsize[3], int comp_order, int backend,
                                        int for_c2r, float scale, void *out);

/* Multiply a real array by scale (e.g. the C2R normalisation). */
pk_status pk_scale_real(void *stream, float *mesh, int64_t size, float scale);

/* One uniform [0, 1) float64 variate per particle id, d_out[i] = jax.random.uniform(
 * fold_in(fold_in(key(seed), lo32(ids[i])), hi32(ids[i])), ()) with jax_enable_x64
 * (Threefry-2x32, 20 rounds): the per-id draw of create_sharded_random((seed, ids))
 * (mesh.py:237-329, _fold_in mesh.py:215-233) that split_particles (mesh.py:3160-3204)
 * uses for disjoint random subsamples of the randoms in compute_fkp2_normalization(split=)
 * (mesh2.py:543).  d_ids NULL: jax.random.uniform(key(seed), (n,)) over the whole array
 * (partitionable Threefry layout, one device), the draw for an integer seed. */
pk_status pk_uniform_ids(void *stream, uint64_t seed, const int64_t *d_ids, int64_t n, double *d_out);

/* --------------------------------------------------------------- binning
 * Bins are the reference's BinMesh2SpectrumPoles (mesh2.py:25-119):
 * k edges edges[0..nedges-1] (float32-rounded, as jnp.digitize compares them),
 * bin b in [0, nedges-1) holds modes with edges[b] <= |k| < edges[b+1]; |k|
 * from kcoords (mesh.py:1605-1636) in float32: kfun[d] * N_d * fftfreq.
 * step > 0 declares uniform edges edges[b] = edges[0] + b*step (fast path).
 * Accumulation: float32 per-mode values, warp-segmented float32 partials,
 * float64 per-CTA histograms, float64 final sum in a fixed order
 * (deterministic).  Outputs are float64. */
pk_status pk_bin_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                size_t *bytes);

/* nmodes[b] = sum of Hermitian weights, ksum[b] = sum of w |k| (mesh.py:2833-2863). */
pk_status pk_bin_modes(void *stream, const int32_t meshsize[3], const float kfun[3],
                       const float *d_edges, int nedges, float step, int backend,
                       double *d_nmodes, double *d_ksum, void *workspace,
                       size_t workspace_bytes);

/* pk_bin_global over nbatch meshes (delta1[b], delta2[b] contiguous) in one launch;
 * d_out[(b * nells + ill) * nbins + bin]; workspace from pk_bin_batch_workspace_size. */
pk_status pk_bin_batch_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                      int nbatch, size_t *bytes);
pk_status pk_bin_global_batch(void *stream, const void *delta1, const void *delta2, int nbatch,
                              const int32_t meshsize[3], const float kfun[3], const float los[3],
                              const float *d_edges, int nedges, float step, int backend,
                              int nells, const int32_t *ells, double *d_out, void *workspace,
                              size_t workspace_bytes);

/* BinMesh2SpectrumPoles.__call__ (mesh2.py:100-119) numerator: per-bin sum of
 * w * value for a complex mesh; d_out[0 * nbins + b] real part,
 * d_out[1 * nbins + b] imaginary part.  remove_zero drops the k = 0 mode. */
pk_status pk_bin_mesh(void *stream, const void *value, const int32_t meshsize[3],
                      const float kfun[3], const float *d_edges, int nedges, float step,
                      int backend, int remove_zero, double *d_out, void *workspace,
                      size_t workspace_bytes);

/* Global line of sight (mesh2.py:346-374): for each requested ell,
 * sum over the bin of w * Re/Im(A) * L_ell(mu), mu = k.los / |k| (|k|(0) = 1),
 * A = |delta1|^2 (delta2 NULL) or conj(delta1) delta2; ell > 0 drops k = 0.
 * Re for even ell, Im for odd.  d_out[ill * nbins + b] (raw sums; divide by
 * nmodes and multiply by 2 ell + 1 on the host). */
pk_status pk_bin_global(void *stream, const void *delta1, const void *delta2,
                        const int32_t meshsize[3], const float kfun[3], const float los[3],
                        const float *d_edges, int nedges, float step, int backend,
                        int nells, const int32_t *ells, double *d_out, void *workspace,
                        size_t workspace_bytes);

/* --------------------------------------------------- correlation function (real space)
 * Binning on the real-space separation grid of BinMesh2CorrelationPoles
 * (mesh2.py:124-192, _make_edges2('real'), mesh2.py:25-62): separation coordinates
 * s_d = fftfreq(n_d)[i] * cellsize_d * n_d on the full real mesh (unit weights), bins of
 * |s| by exact |s|^2 thresholds as for k.  Workspace from pk_bin_separation_workspace_size. */
pk_status pk_bin_separation_workspace_size(const int32_t meshsize[3], int nedges, int nvalues,
                                           size_t *bytes);

/* Per-bin number of separations (d_nmodes) and sum of |s| (d_ssum), float64. */
pk_status pk_bin_separation_modes(void *stream, const int32_t meshsize[3], const float cellsize[3],
                                  const float *d_edges, int nedges, float step, double *d_nmodes,
                                  double *d_ssum, void *workspace, size_t workspace_bytes);

/* Fixed line of sight branch of compute_mesh2_correlation (mesh2.py:465-499): for each
 * multipole ell (nells <= 3) the per-bin sum of value(s) L_ell(mu), mu = s.los / |s|
 * (|s| = 1 at s = 0), the s = 0 cell dropped for ell > 0; value is a real mesh (float32,
 * e.g. c2r(|delta_k|^2)).  d_out: (nells, nbins) float64 sums (divide by nmodes,
 * times 2 ell + 1). */
pk_status pk_bin_separation_global(void *stream, const float *value, const int32_t meshsize[3],
                                   const float cellsize[3], const float los[3], const float *d_edges,
                                   int nedges, float step, int nells, const int32_t *ells,
                                   double *d_out, void *workspace, size_t workspace_bytes);

/* Mode oversampling of BinMesh2CorrelationPoles (mode_oversampling > 0, _make_edges2('real'),
 * mesh2.py:48-61): the separations binned by |s + sshift| (sshift added to each coordinate in
 * float32, as the reference adds its integer shifts), their values and mu from s; one call per
 * shift, written or added (accumulate) into the outputs, the caller averaging over the shifts. */
pk_status pk_bin_separation_modes_shifted(void *stream, const int32_t meshsize[3], const float cellsize[3],
                                          const float sshift[3], const float *d_edges, int nedges, float step,
                                          int accumulate, double *d_nmodes, double *d_ssum, void *workspace,
                                          size_t workspace_bytes);
pk_status pk_bin_separation_global_shifted(void *stream, const float *value, const int32_t meshsize[3],
                                           const float cellsize[3], const float sshift[3], const float los[3],
                                           const float *d_edges, int nedges, float step, int nells,
                                           const int32_t *ells, int accumulate, double *d_out, void *workspace,
                                           size_t workspace_bytes);

/* Spherical-Bessel basis of BinMesh2CorrelationPoles (basis='bessel', mesh2.py:169-181),
 * for the estimators of compute_mesh2_correlation (mesh2.py:414-500): per separation bin b
 * (s_b = d_sep[b], float64, the bins' xavg) and multipole ells[l] the float64 sum over the
 * stored modes (each once, no Hermitian weight) of Re(A_l(k)) j_ell(|k| s_b), |k| and
 * |k| s_b in float32, j_ell in float64.  A_l is |d1|^2 or conj(d1) d2 times L_ell(mu)
 * (los given, ell <= 4), or, with los NULL (first point), |A0|^2 / conj(B0) A0 for ell 0
 * (d1 = A0, d2 = B0 or NULL; when include_ell0) and conj(sum_t F_t Y_t(khat)) A0 over this
 * call's terms (f: nterms half-complex meshes) for ell > 0; k = 0 is dropped for ell > 0.
 * klimit (NULL: none): only klimit[0] <= |k| < klimit[1].  d_out: (nells, nbins), written or,
 * with accumulate, added to; multiply by (-1)^(ell/2) / N and the estimator's factor.
 * nbins <= 1024, nells <= 5.  Workspace from pk_bin_bessel_workspace_size. */
pk_status pk_bin_bessel_workspace_size(const int32_t meshsize[3], int nbins, int nells, size_t *bytes);
pk_status pk_bin_bessel(void *stream, const void *d1, const void *d2, const void *f, int nterms,
                        const int32_t *term_ell, const int32_t *term_m, const int32_t meshsize[3],
                        const float kfun[3], int backend, const float *los, const double *d_sep, int nbins,
                        const float *klimit, int nells, const int32_t *ells, int include_ell0,
                        int accumulate, double *d_out, void *workspace, size_t workspace_bytes);

/* Window matrix of the global line-of-sight power spectrum, mesh input power
 * (compute_mesh2_spectrum_window, mesh2.py:1013-1133).  'jax' (rfftn) layout only.
 *
 * pk_window_fill: ncolumns (<= 16) half-complex meshes, column c at out + c N_c:
 *   scale * L_ellin(mu) + 0i where klo[c] <= |k| < khi[c], 0 elsewhere (mesh2.py:1123),
 *   |k| = sqrt((kx^2 + ky^2) + kz^2), mu = k.los / |k| (|k| = 1 at k = 0), float32.
 * pk_window_multiply: meshes[c n + i] *= q[i] for c < ncolumns (16-byte aligned buffers);
 *   the real-space product Q * c2r(A) of mesh2.py:1124.
 * pk_bin_window: per bin and output multipole the float64 sum of w Re(A) L_ell(mu) over the
 *   stored modes, k = 0 dropped for every ell, odd ell 0 (the reference bins
 *   A (L_ell(mu) + L_ell(-mu))); A is `value` (half-complex, complex64) or, when value is
 *   NULL, the periodic column scale * L_ellin(mu) 1{klo <= |k| < khi} formed per mode.
 *   d_out: (nells, nbins); divide by nmodes and multiply by (2 ell + 1) / N. */
pk_status pk_window_fill(void *stream, const int32_t meshsize[3], const float kfun[3], int backend,
                         const float los[3], int ellin, float scale, int ncolumns, const float *klo,
                         const float *khi, void *out);
pk_status pk_window_multiply(void *stream, float *meshes, int ncolumns, const float *q, int64_t n);
pk_status pk_bin_window(void *stream, const void *value, const int32_t meshsize[3], const float kfun[3],
                        const float los[3], const float *d_edges, int nedges, float step, int backend,
                        int nells, const int32_t *ells, int ellin, float klo, float khi, float scale,
                        double *d_out, void *workspace, size_t workspace_bytes);

/* Selection-function window columns and mean spectra (compute_mesh2_spectrum_mean,
 * mesh2.py:1569-1605), nbatch (<= 65535) half-complex meshes A (value + b N_c): per mesh, bin
 * and even ell (nells <= 5) the float64 sum of w Re(A) L_ell(mu) over the stored modes, k = 0
 * dropped when remove_zero (the fused global-los binning pass, linear in A).  Odd ell rows
 * are zero in both (L_ell(mu) + L_ell(-mu) = 0) and are not asked for.  workspace:
 * pk_bin_batch_workspace_size(meshsize, nedges, nells, nbatch).  d_out: (nbatch, nells, nbins). */
pk_status pk_bin_window_batch(void *stream, const void *value, int nbatch, const int32_t meshsize[3],
                              const float kfun[3], const float los[3], const float *d_edges, int nedges,
                              float step, int backend, int nells, const int32_t *ells, int remove_zero,
                              double *d_out, void *workspace, size_t workspace_bytes);

/* First-point mean spectrum (compute_mesh2_spectrum_mean, mesh2.py:1607-1669).
 * pk_ylm_kgrid_multiply: for nterms (<= 32) real Y_lm, out_t (+)= scale value(k) Y_t(khat) on
 *   the half-complex 'jax' grid (khat = k / |k|, 0 at k = 0; out_t at out + t N_c).
 * pk_sum_products: out[i] (+)= sum_t coef[t] a[t n + i] b[t n + i] over nterms (<= 32) pairs of
 *   real meshes (the Q = sum 4 pi / (2 ell1 + 1) xi G of mesh2.py:1641-1644). */
pk_status pk_ylm_kgrid_multiply(void *stream, const void *value, const int32_t meshsize[3], const float kfun[3],
                                int nterms, const int32_t *term_ell, const int32_t *term_m, float scale,
                                int accumulate, void *out);
pk_status pk_sum_products(void *stream, float *out, const float *a, const float *b, int nterms, const float *coef,
                          int64_t n, int accumulate);

/* Periodic window, all columns of disjoint input bins in one pass: d_edges (nedges, float32,
 * ascending) is the union of the output and input edges; for each of npairs (<= 9) pairs
 * (pair_ell, pair_ellin) the float64 sum per merged interval of
 * w scale L_ellin(mu) L_ell(mu) (k = 0 dropped, odd ell 0).  Each merged interval lies in
 * one output bin and at most one input bin; the caller adds the intervals into the window.
 * d_out: (npairs, nedges - 1). */
pk_status pk_bin_window_pairs(void *stream, const int32_t meshsize[3], const float kfun[3], const float los[3],
                              const float *d_edges, int nedges, float step, int backend, int npairs,
                              const int32_t *pair_ell, const int32_t *pair_ellin, float scale, double *d_out,
                              void *workspace, size_t workspace_bytes);

/* First-point correlation function (mesh2.py:423-451): carry += sum_j r_j Y_j(shat) over
 * nterms real meshes r_j (r + j N_r), shat the unit separation vector of the grid
 * fftfreq(n) * cellsize * n (0 at s = 0), real Y_lm as pk_ylm_premultiply. */
pk_status pk_ylm_separation_accumulate(void *stream, const float *r, const int32_t meshsize[3],
                                       const float cellsize[3], int nterms, const int32_t *term_ell,
                                       const int32_t *term_m, float *carry);

/* out_t = conj(f_t) * a for nterms complex meshes f_t (f + t n) of n complex64 values each
 * (the conj(F) A0 products of the first-point estimators). */
pk_status pk_conj_multiply(void *stream, const void *f, const void *a, int nterms, int64_t n, void *out);

/* Wide-angle orders of the first-point window matrix (mesh2.py:1214, 1249, 1273) and mean
 * spectrum (mesh2.py:1644-1645): mesh_b *= |x|^power (separation = 0: x the cell-corner
 * position offset + i cellsize, as in pk_ylm_premultiply) or |s|^power (separation = 1: the
 * separation grid of pk_ylm_separation_accumulate), for nmeshes consecutive real meshes;
 * |power| <= 8, negative powers as 1 / |x|^-power. */
pk_status pk_radial_power(void *stream, float *mesh, int nmeshes, const int32_t meshsize[3],
                          const float cellsize[3], const float offset[3], int separation, int power);

/* pk_bin_global_batch of the meshes that pk_interlace_compensate(_batch) would form
 * (for_c2r = 0, scale 1), without storing them: each mode is combined on the fly from
 * the nshifts interlaced, uncompensated R2C meshes (shifted: nbatch x nshifts Hermitian
 * meshes, mesh s of batch b at shifted + (b * nshifts + s) * N_c) with compensation
 * order comp_order, then binned.  Same outputs and workspace as pk_bin_global_batch.
 * Takes up to 3 even multipoles (ell <= 4) and up to 4 shifts (PK_ERR_RANGE otherwise).
 * No reference counterpart: the reference stores the combined mesh (mesh.py:2737-2752)
 * and then bins it (mesh2.py:346-374). */
pk_status pk_bin_global_interlaced(void *stream, const void *shifted, int nbatch, int nshifts,
                                   int comp_order, const int32_t meshsize[3], const float kfun[3],
                                   const float los[3], const float *d_edges, int nedges, float step,
                                   int backend, int nells, const int32_t *ells, double *d_out,
                                   void *workspace, size_t workspace_bytes);

/* Mode oversampling of BinMesh2SpectrumPoles (mode_oversampling = s > 0, mesh2.py:48-61,
 * _bincount mesh.py:2876-2910): the reference bins the modes once per integer shift in
 * [-s, s]^3 by |k + shift| (the shift added to each k coordinate in float32; Hermitian
 * weights and the binned values of k unchanged) and averages the per-shift sums.  Each call
 * below is one shift (kshift = the shift as float32), the counterpart of pk_bin_modes /
 * pk_bin_mesh / pk_bin_global / pk_bin_firstpoint with the bin of |k + kshift|; with
 * `accumulate` it adds into the outputs, so the caller sums the (2s+1)^3 calls and divides.
 * Same workspaces as the unshifted entry points. */
pk_status pk_bin_modes_shifted(void *stream, const int32_t meshsize[3], const float kfun[3], const float kshift[3],
                               const float *d_edges, int nedges, float step, int backend, int accumulate,
                               double *d_nmodes, double *d_ksum, void *workspace, size_t workspace_bytes);
pk_status pk_bin_mesh_shifted(void *stream, const void *value, const int32_t meshsize[3], const float kfun[3],
                              const float kshift[3], const float *d_edges, int nedges, float step, int backend,
                              int remove_zero, int accumulate, double *d_out, void *workspace,
                              size_t workspace_bytes);
pk_status pk_bin_global_shifted(void *stream, const void *delta1, const void *delta2, const int32_t meshsize[3],
                                const float kfun[3], const float kshift[3], const float los[3], const float *d_edges,
                                int nedges, float step, int backend, int nells, const int32_t *ells, int accumulate,
                                double *d_out, void *workspace, size_t workspace_bytes);
pk_status pk_bin_firstpoint_shifted(void *stream, const void *a0, const void *b0, const void *f, int nterms,
                                    const int32_t *term_ell, const int32_t *term_m, const int32_t meshsize[3],
                                    const float kfun[3], const float kshift[3], const float *d_edges, int nedges,
                                    float step, int backend, int nells, const int32_t *ells, int include_ell0,
                                    int accumulate, double *d_out, void *workspace, size_t workspace_bytes);

/* No counterpart in the reference.  pk_bin_global without a workspace argument, for
 * callers that cannot allocate device memory when they call (a host callback, or a
 * foreign runtime that owns the allocator): its scratch is a fixed 16 MiB static device
 * array, held by every GPU that loads the library until exit.  Returns PK_ERR_RANGE when
 * the bins x multipoles need more scratch than that.  The first call on a device looks
 * the array's address up (make it before any stream capture); later calls on a stream
 * that is not capturing look it up again, so a recreated context (cudaDeviceReset) is
 * picked up.  Calls that overlap on the GPU share the array and race. */
pk_status pk_bin_global_noalloc(void *stream, const void *delta1, const void *delta2,
                                const int32_t meshsize[3], const float kfun[3],
                                const float los[3], const float *d_edges, int nedges, float step,
                                int backend, int nells, const int32_t *ells, double *d_out);

/* First-point line of sight (mesh2.py:293-344), one batch of (ell, m) terms:
 * d_out[ill * nbins + b] (+)= sum over the bin of w * Re/Im(conj(S_ell) A0),
 * S_ell = sum_{m in batch} F_j(k) Y_ell,m(khat), F_j = r2c(rho Y_ell,m(xhat)).
 * ell = 0 entries of `ells` take |A0|^2 (or conj(B0) A0 with b0 != NULL) and
 * are only accumulated when include_ell0 != 0.  accumulate != 0 adds into d_out. */
pk_status pk_bin_firstpoint(void *stream, const void *a0, const void *b0, const void *f,
                            int nterms, const int32_t *term_ell, const int32_t *term_m,
                            const int32_t meshsize[3], const float kfun[3],
                            const float *d_edges, int nedges, float step, int backend,
                            int nells, const int32_t *ells, int include_ell0,
                            int accumulate, double *d_out, void *workspace,
                            size_t workspace_bytes);

/* Real-space Y_lm premultiply for the first-point estimator (mesh2.py:313-327):
 * out[j] = rho(x) * Y_{ell_j, m_j}(xhat) at cell corners
 * x_i = i * cellsize + (boxcenter - boxsize/2) (mesh.py:1594-1603), observer at 0. */
pk_status pk_ylm_premultiply(void *stream, const float *rho, const int32_t meshsize[3],
                             const float cellsize[3], const float offset[3], int nterms,
                             const int32_t *term_ell, const int32_t *term_m, float *out);

/* ----------------------------------------------------------------- adjoints
 * Hand-written backward passes (the reference differentiates this path with JAX
 * autodiff: the transpose of the scatter is resamplers.read, resamplers.py:100-125, FFT
 * adjoints come from XLA).  Conjugate cotangents are dL/dRe + i dL/dIm.  With
 * for_c2r / from_real the Fourier-space cotangents are converted so that an
 * unnormalised C2R yields the cotangent of the real mesh they were transformed from.
 * Odd multipoles of auto spectra are identically zero and carry no gradient. */
pk_status pk_adjoint_workspace_size(int nedges, size_t *bytes);

/* Backward of pk_bin_global for an auto spectrum: out = 2 G delta with
 * G = w_k sum_l coef[l * nbins + b] L_l(mu); coef is float32 (nells, nbins). */
pk_status pk_bin_global_adjoint(void *stream, const void *delta, const int32_t meshsize[3],
                                const float kfun[3], const float los[3], const float *d_edges,
                                int nedges, float step, float edge0, int backend, int nells,
                                const int32_t *ells, const float *d_coef, int for_c2r, void *out,
                                void *workspace, size_t workspace_bytes);

/* Backward of pk_bin_firstpoint (auto): cotangents of A0 (written or accumulated) and
 * of each F_j of the batch (out_f[j]).  Even ells bin Re(conj(S) A0), odd ells
 * Im(conj(S) A0) (mesh2.py:334).  for_c2r = 2 converts the F_j cotangents for C2R but
 * leaves the A0 cotangent as the conjugate cotangent of a complex input mesh. */
pk_status pk_bin_firstpoint_adjoint(void *stream, const void *a0, const void *f, int nterms,
                                    const int32_t *term_ell, const int32_t *term_m,
                                    const int32_t meshsize[3], const float kfun[3],
                                    const float *d_edges, int nedges, float step, float edge0,
                                    int backend, int nells, const int32_t *ells,
                                    const float *d_coef, int for_c2r, void *out_a0,
                                    int accumulate_a0, void *out_f, void *workspace,
                                    size_t workspace_bytes);

/* pk_bin_global_adjoint / pk_bin_firstpoint_adjoint for mode oversampling (mesh2.py:48-61,
 * the forward through the *_shifted binning calls): nkshift (<= 125) k shifts, kshifts
 * (host, 3 floats each, as given to those calls); each mode's coefficient is the mean over the
 * shifts of coef[l][bin of |k + shift|]. */
pk_status pk_bin_global_adjoint_shifted(void *stream, const void *delta, const int32_t meshsize[3],
                                        const float kfun[3], const float los[3], const float *d_edges,
                                        int nedges, float step, float edge0, int backend, int nells,
                                        const int32_t *ells, const float *d_coef, int for_c2r, int nkshift,
                                        const float *kshifts, void *out, void *workspace,
                                        size_t workspace_bytes);
pk_status pk_bin_firstpoint_adjoint_shifted(void *stream, const void *a0, const void *f, int nterms,
                                            const int32_t *term_ell, const int32_t *term_m,
                                            const int32_t meshsize[3], const float kfun[3],
                                            const float *d_edges, int nedges, float step, float edge0,
                                            int backend, int nells, const int32_t *ells, const float *d_coef,
                                            int for_c2r, int nkshift, const float *kshifts, void *out_a0,
                                            int accumulate_a0, void *out_f, void *workspace,
                                            size_t workspace_bytes);

/* Backward of pk_interlace_compensate (mesh.py:2737-2752), either backend's phases: from the
 * cotangent of the combined mesh (R = rfftn(rho_bar) if from_real, else the conjugate
 * cotangent of the complex mesh) to nshifts Hermitian half-meshes whose unnormalised C2R
 * are the cotangents of the painted shifted meshes. */
pk_status pk_interlace_adjoint(void *stream, const void *in, int from_real, int nshifts,
                               const int32_t meshsize[3], int comp_order, int backend, void *out);

/* Backward of the normalised C2R (jnp.fft.irfftn, mesh.py:1699-1719) of a Hermitian
 * half-mesh: out (+)= R w_z / (N0 N1 N2), R = rfftn(rho_bar), w_z = 2 off the kz = 0 and
 * kz = N2/2 planes, 1 on them: the conjugate cotangent of the complex mesh.  No
 * reference counterpart (JAX transposes its FFTs itself). */
pk_status pk_c2r_adjoint(void *stream, const void *r, const int32_t meshsize[3], int accumulate,
                         void *out);

/* Backward of pk_ylm_premultiply: rho_bar += sum_j r_j Y_j(xhat). */
pk_status pk_ylm_accumulate(void *stream, const float *r, const int32_t meshsize[3],
                            const float cellsize[3], const float offset[3], int nterms,
                            const int32_t *term_ell, const int32_t *term_m, float *rho_bar);

/* ---- learned aliasing correction: BF16 MLP (16 -> 128 -> 128 -> 128 -> 1, SiLU) ----
 * No counterpart in the reference (the learned correction is a new method).  Parameters
 * are one flat float32 array of pk_mlp_num_params() entries (W0 [128][16], b0 [128],
 * W1 [128][128], b1, W2 [128][128], b2, W3 [8][128] (row 0 used), b3 [8] (entry 0 used))
 * and its bf16 copy in the same layout; matrices are row-major (out x in).  Inputs are
 * float32 rows of 16 features; idx (may be NULL) gathers the rows / targets of a batch. */
int pk_mlp_num_params(void);

/* wb = bf16(w), round to nearest even. */
pk_status pk_mlp_cast(void *stream, const float *w, void *wb);

/* y[i] = MLP(x[idx[i]]), bf16 operands with float32 accumulation, float32 biases.  With
 * z and h (float32 [3][batch][128]) also stores the hidden pre-activations / activations
 * for pk_mlp_backward. */
pk_status pk_mlp_forward(void *stream, const float *x, const int32_t *idx, int batch, const void *wb,
                         const float *w, float *y, float *z, float *h);

/* pk_mlp_forward on the 5th-generation tensor cores (tcgen05.mma, bf16 operands in shared
 * memory, float32 accumulators in tensor memory), 128 samples per CTA.  Same inputs and
 * outputs as pk_mlp_forward (wb 16-byte aligned).  d_status (device int, may be NULL) is
 * set to 1 if a tensor-core step did not complete within its bounded wait. */
pk_status pk_mlp_forward_tc(void *stream, const float *x, const int32_t *idx, int batch, const void *wb,
                            const float *w, float *y, float *z, float *h, int32_t *d_status);

/* Weighted MSE: loss = sum_i w_j (y_i - t_j)^2 / batch with j = idx[i]; dy = dloss/dy.
 * weight and loss may be NULL. */
pk_status pk_mlp_mse(void *stream, const float *y, const float *target, const float *weight,
                     const int32_t *idx, int batch, float *dy, float *loss);

pk_status pk_mlp_backward_workspace_size(int batch, size_t *bytes);

/* grad = d(sum_i dy_i y_i)/d(params) from the stored z, h (deterministic: per-CTA partial
 * gradients added in a fixed order). */
pk_status pk_mlp_backward(void *stream, const float *x, const int32_t *idx, int batch, const void *wb,
                          const float *z, const float *h, const float *dy, float *grad,
                          void *workspace, size_t workspace_bytes);

/* pk_mlp_backward on the 5th-generation tensor cores: dW_l += bf16(dZ_l)^T bf16(A_l) and
 * dH_{l-1} = bf16(dZ_l) bf16(W_l) as tcgen05.mma with float32 accumulators in tensor memory
 * (the weight gradients accumulate there over a persistent CTA's 128-sample tiles), bias and
 * output-layer gradients as fixed-order float32 column sums; one partial row per CTA (at most
 * one CTA per SM), added in CTA order.  The same workspace as pk_mlp_backward suffices; wb, z
 * and h 16-byte aligned.  d_status (device int, may be NULL) is set to 1 if a tensor-core step
 * did not complete within its bounded wait. */
pk_status pk_mlp_backward_tc(void *stream, const float *x, const int32_t *idx, int batch, const void *wb,
                             const float *z, const float *h, const float *dy, float *grad,
                             void *workspace, size_t workspace_bytes, int32_t *d_status);

/* AdamW step on w (and its bf16 copy wb): t = *step (device int, steps taken so far),
 * learning rate lr_table[min(t, ntable - 1)] (device), bias corrections 1 - beta^(t + 1),
 * then *step = t + 1.  Everything the step depends on lives on the device, so a captured
 * CUDA graph of training steps replays with a learning-rate schedule. */
pk_status pk_mlp_adam(void *stream, float *w, void *wb, float *m, float *v, const float *grad,
                      const float *lr_table, int ntable, int32_t *step, float beta1, float beta2,
                      float eps, float weight_decay);

#ifdef __cplusplus
}
#endif

#endif /* JAXPOWER_B200_H */
