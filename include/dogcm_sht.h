/*
 * dogcm_sht.h -- C-ABI of the B200 spherical-harmonic transform library
 * (libdogcm_sht.so).
 *
 * It replaces the horizontal part of dogcm's spectral utility module
 * model/dogcm/src/util/math/SpmlUtil_mod.f90 (and the SPMODEL wa_module
 * routines that module re-exports at SpmlUtil_mod.f90:105-135).  Every entry
 * point cites the reference routine it stands in for.  A Fortran host binds
 * these through ISO_C_BINDING.
 *
 * Conventions
 *  - All arrays are FP64 and use the reference's Fortran layouts:
 *      grid      xya(0:im-1, 1:jm, nb)  lon fastest, Gauss latitudes
 *                ascending from the south pole;
 *      spectral  wa(lm, nb), lm = (nm+1)^2, l_nm(n,m) = n(n+1)+m+1 (1-based).
 *                wa(l_nm(n,0)) = a_n^0.  For m > 0, wa(l_nm(n,m)) = sqrt2 Re a_n^m
 *                and wa(l_nm(n,-m)) = sqrt2 Im a_n^m, for the field
 *                sum_n sum_m a_n^m Pbar_n^|m|(mu) e^{i m lambda}, where
 *                int_{-1}^{1} Pbar^2 dmu = 2.
 *    nb is the number of field-levels (the trailing dimension).  nb = 1 is the
 *    single-level form (w_xy, xy_w, ...), nb = km the wa_/xya_ form.
 *  - Every function returns an int status (SHT_OK = 0).  The reference
 *    aborts through MessageNotify('E', ...) on misuse.  Here the caller maps a
 *    nonzero status to that abort, and sht_last_error() gives the message.
 *  - Functions without a suffix take HOST pointers and return when the
 *    results are in host memory.  The *_dev variants take DEVICE pointers and
 *    are ordered on the plan's stream (sht_set_stream).  They return once the
 *    work is enqueued.
 *  - Calls on one plan are serialised internally: the plan owns its device
 *    workspace.  Different plans may be used from different host threads.
 *  - There is no CPU fallback.  Without a usable CUDA device every compute
 *    entry point returns SHT_ERR_CUDA or SHT_ERR_NO_DEVICE.
 */
#ifndef DOGCM_SHT_H
#define DOGCM_SHT_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SHT_API __attribute__((visibility("default")))
#else
#define SHT_API
#endif

/* ---------------------------------------------------------------- status */
#define SHT_OK                   0
#define SHT_ERR_INVALID_ARG      1  /* null pointer, nb < 0, bad mode            */
#define SHT_ERR_UNSUPPORTED_SIZE 2  /* grid the kernels do not cover (see sht_init) */
#define SHT_ERR_NOT_INITIALIZED  3  /* plan is NULL or already finalised         */
#define SHT_ERR_CUDA             4  /* a CUDA runtime call failed                */
#define SHT_ERR_NO_DEVICE        5  /* no CUDA device visible                    */
#define SHT_ERR_ALLOC            6  /* device or host allocation failed          */
#define SHT_ERR_DEVICE_TIMEOUT   7  /* a bounded device-side wait ran out        */
#define SHT_ERR_TOO_LARGE        8  /* request exceeds a fixed capacity          */

/* precision modes of the Legendre contraction */
#define SHT_PREC_FP64  0  /* FP64 operands and FP64 products (the FP64 tensor
                             path, mma.sync f64), FP64 accumulation            */
#define SHT_PREC_SPLIT 1  /* FP64 operands as signed 8-bit digits (eight per
                             grid or spectral value, seven per table value),
                             exact integer digit products on the tcgen05
                             tensor cores, FP64 recombination                  */
#define SHT_PREC_AUTO  2  /* per direction, the faster of the two on B200 as
                             measured: split precision for a contraction of at
                             least 128 terms (analysis: jm/2 latitudes;
                             synthesis: (nm+3)/2 degrees of one parity), FP64
                             below.  Both meet the same 1e-11 bound.            */

typedef struct sht_plan_s sht_plan;

/* Status text of a code, and the message of the last failure on this thread. */
SHT_API const char *sht_status_string(int status);
SHT_API const char *sht_last_error(void);

/* ------------------------------------------------------------- plan/admin */

/* SpmlUtil_Init(iMax, jMax, kMax, nMax, tMax, RPlanet, np)
 * (SpmlUtil_mod.f90:192-241; wa_Initial at :218-223).
 * im: longitudes (even, 16..2048: powers of two take the four-step FFT, other
 * counts such as 96, 192, 320 or 640 a direct summation over longitudes),
 * or 1 for the axisymmetric model
 * (DOGCM_MODE_AXISYM, SpmlUtil_mod.f90:30-35,210-211: SPMODEL
 * wa_zonal_module, only the m = 0 modes, lm = nm + 1 with wa(n+1) = a_n^0);
 * jm: Gauss latitudes (even); km: levels (the default batch; informational);
 * nm: triangular truncation (nm = -1 selects (im-1)/3, or (2 jm - 1)/3 when
 * im = 1, as util/grid/DOGCM_GaussSpmVFvmGrid_mod.f90:206-209 does);
 * radius: planetary radius (Radius in SpmlUtil_mod).  Requires
 * im >= 2 nm + 2 (unless im = 1) and jm > nm.  Builds the Gauss nodes and
 * weights and the associated-Legendre table on the device in FP64. */
SHT_API int sht_init(int im, int jm, int km, int nm, double radius, sht_plan **plan);

/* SpmlUtil_Final (SpmlUtil_mod.f90:243-256).  Frees the plan. */
SHT_API int sht_final(sht_plan *plan);

/* isInitialzed (SpmlUtil_mod.f90:262-267). 1 if the plan is live. */
SHT_API int sht_is_initialized(const sht_plan *plan);

/* Grid sizes: im, jm, nm and lm = (nm+1)^2.  Any pointer may be NULL. */
SHT_API int sht_dims(const sht_plan *plan, int *im, int *jm, int *nm, int *lm);

/* get_SpmlGridInfo (SpmlUtil_mod.f90:271-295): x_Lon (im), y_Lat (jm, radians),
 * x_Lon_Weight (im, sums to 2 pi), y_Lat_Weight (jm, sums to 2).
 * Any output may be NULL. */
SHT_API int sht_grid_info(const sht_plan *plan, double *x_lon, double *y_lat,
                  double *x_lon_weight, double *y_lat_weight);

/* l_nm / nm_l (re-exported at SpmlUtil_mod.f90:120): 1-based spectral index. */
SHT_API int sht_l_nm(int n, int m);
SHT_API int sht_nm_l(int l, int *n, int *m);

/* The same maps for the plan's layout (the axisymmetric layout is l = n + 1,
 * m = 0); sht_plan_l_nm returns 0 for a pair the plan does not hold. */
SHT_API int sht_plan_l_nm(const sht_plan *plan, int n, int m);
SHT_API int sht_plan_nm_l(const sht_plan *plan, int l, int *n, int *m);

/* rn(:,1) (SpmlUtil_mod.f90:135): Laplacian eigenvalue -n(n+1) per l. */
SHT_API int sht_rn(const sht_plan *plan, double *rn);

/* Precision of the Legendre contraction for the following calls:
 * SHT_PREC_FP64 (the default), SHT_PREC_SPLIT or SHT_PREC_AUTO. */
SHT_API int sht_set_precision(sht_plan *plan, int mode);
SHT_API int sht_get_precision(const sht_plan *plan, int *mode);

/* Kernel choices (used by the autotuner and the tests; the defaults are
 * picked per grid).  SHT_OPT_LEGENDRE_KERNEL: 0 automatic, 1 per-band kernel
 * (any grid), 2 persistent paired-band kernel (T85 and smaller), 3 persistent
 * latitude-chunked paired-band kernel (jm/2 a multiple of 16, up to T341),
 * 4 the whole plain analysis or synthesis (w_xy, xy_w and their batched
 * forms) in one kernel per call, Fourier coefficients kept on chip (power-of-
 * two im <= 128, jm/2 a multiple of 4, FP64; other operators keep the
 * automatic kernels; the automatic choice for im = 32).  A choice that does
 * not cover the grid falls back to the automatic one. */
#define SHT_OPT_LEGENDRE_KERNEL 1
/* SHT_OPT_HOST_GRAPHS: 1 (default) replays small host-pointer calls (those
 * staged through the plan's page-locked buffer) as CUDA graphs from the
 * second call of an operator and size on; 0 launches every call directly.
 * Either way the results are identical.  SHT_OPT_HOST_GRAPH_COUNT (read only)
 * is the number of graphs the plan holds. */
#define SHT_OPT_HOST_GRAPHS 2
#define SHT_OPT_HOST_GRAPH_COUNT 3
/* SHT_OPT_LEGENDRE_TILE: the tile of the FP64 Legendre kernels (0 automatic).
 * Paired kernels: 8 or 16 complex columns per analysis item; chunked kernels:
 * 16 or 32 latitudes per streamed chunk.  A value the chosen kernel does not
 * take, or whose shared memory does not fit, falls back to the automatic
 * tile.  Results are identical for every tile (the same products in the same
 * order per output).  The batch tuner (sht_multi_build with autotune) times
 * the tiles with the kernel families. */
#define SHT_OPT_LEGENDRE_TILE 4
SHT_API int sht_set_option(sht_plan *plan, int option, int value);
SHT_API int sht_get_option(const sht_plan *plan, int option, int *value);

/* Self-test of the device-side failure path: one block waits, through the
 * bounded wait the split-precision kernel uses, on a shared-memory barrier
 * that nothing arrives at, gives up after limit_ms milliseconds (1..1000)
 * and records the timeout in the plan's device error word.  Returns what the
 * status check after a synchronous call then reports:
 * SHT_ERR_DEVICE_TIMEOUT when the bound and the error word work.  The word is
 * cleared and the plan stays usable.  No counterpart in the reference (its
 * failures abort through MessageNotify).  Grids outside the split kernel
 * return SHT_ERR_UNSUPPORTED_SIZE. */
SHT_API int sht_selftest_device_timeout(sht_plan *plan, int limit_ms);

/* Stream for the *_dev calls (a cudaStream_t passed as void*; NULL = legacy
 * default stream), and a wait for all work on it. */
SHT_API int sht_set_stream(sht_plan *plan, void *stream);
SHT_API int sht_synchronize(sht_plan *plan);

/* ------------------------------------------------- transforms, host arrays */

/* w_xy / wa_xya / wz_xyz: grid -> spectral analysis
 * (SPMODEL wa_module via SpmlUtil_mod.f90:110; wz_xyz alias at
 * model/old/sogcm/util/SpmlUtil_mod.f90:323-333). */
SHT_API int sht_wa_xya(sht_plan *plan, const double *xya, int nb, double *wa);

/* xy_w / xya_wa / xyz_wz: spectral -> grid synthesis (SpmlUtil_mod.f90:110;
 * model/old/sogcm/util/SpmlUtil_mod.f90:308-320). */
SHT_API int sht_xya_wa(sht_plan *plan, const double *wa, int nb, double *xya);

/* w_DivLambda_xy: spectral of (1/(1-mu^2)) dA/dlambda (SpmlUtil_mod.f90:116). */
SHT_API int sht_wa_divlambda_xya(sht_plan *plan, const double *xya, int nb, double *wa);

/* w_DivMu_xy: spectral of dB/dmu (SpmlUtil_mod.f90:116). */
SHT_API int sht_wa_divmu_xya(sht_plan *plan, const double *xya, int nb, double *wa);

/* xy_GradLambda_w (d/dlambda), xy_GradMu_w ((1-mu^2) d/dmu),
 * xy_GradLon_w ((1/cos phi) d/dlambda), xy_GradLat_w (d/dphi)
 * (SpmlUtil_mod.f90:114-115). */
SHT_API int sht_xya_gradlambda_wa(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradmu_wa(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradlon_wa(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradlat_wa(sht_plan *plan, const double *wa, int nb, double *xya);

/* w_AlphaOptr_xy / wa_AlphaOptr_xya: (DivLambda(A) + DivMu(B)) / a
 * (SpmlUtil_mod.f90:398-412, 453-473). */
SHT_API int sht_wa_alphaoptr_xya(sht_plan *plan, const double *xya_a, const double *xya_b,
                         int nb, double *wa);

/* xy_AlphaOptr_w / xya_AlphaOptr_wa: (GradLambda(A) + GradMu(B)) / (a cos^2 phi)
 * (SpmlUtil_mod.f90:414-451). */
SHT_API int sht_xya_alphaoptr_wa(sht_plan *plan, const double *wa_a, const double *wa_b,
                         int nb, double *xya);

/* w_AlphaOptr_xy(A Q, B Q) with the point-by-point products formed inside the
 * longitude transform: the horizontal tracer flux divergence of the thickness
 * equation, where Q = H cos(phi) T multiplies both velocity components
 * (dynamics/hspm_vfvm/HBEBaroc_hspm_vfvm_mod.f90:160-165).  xya_q holds one grid per level, like
 * xya_a and xya_b. */
SHT_API int sht_wa_alphaoptr_prod_xya(sht_plan *plan, const double *xya_a, const double *xya_b,
                              const double *xya_q, int nb, double *wa);

/* xy_GradLon_w and xy_GradLat_w of the same spectrum in one synthesis
 * (SpmlUtil_mod.f90:114-115): both gradients share the staged spectral
 * entries and the Legendre and longitude passes run over 2 nb columns. */
SHT_API int sht_xya_hgrad_wa(sht_plan *plan, const double *wa, int nb, double *xya_lon,
                     double *xya_lat);

/* The Redi/GM tracer gradients, xy_GradLon_w(w_xy(T)) and
 * xy_GradLat_w(w_xy(T)) (physics/lphys/LPhys_RediGM_hspm_vfvm_mod.f90:432-440),
 * grid to grid without a spectral array on the caller's side.  Like the
 * SPMODEL functions, no 1/radius factor is applied. */
SHT_API int sht_xya_hgrad_xya(sht_plan *plan, const double *xya, int nb, double *xya_lon,
                      double *xya_lat);

/* xy_w(w_AlphaOptr_xy(A, B)) grid to grid: the divergence of the Redi/GM
 * tracer fluxes added to the tendency (physics/lphys/
 * LPhys_RediGM_hspm_vfvm_mod.f90:350-355, A and B the flux components times
 * cos(phi)).  One analysis of 2 nb columns into a device temp, then one
 * synthesis; no spectral array on the caller's side. */
SHT_API int sht_xya_fluxdiv_xya(sht_plan *plan, const double *xya_a, const double *xya_b, int nb,
                        double *xya);

/* calc_UVCosLat2VorDiv: Vor = H(V cos, -U cos), Div = H(U cos, V cos)
 * (SpmlUtil_mod.f90:299-314, 342-368). Inputs are U cos phi and V cos phi. */
SHT_API int sht_uvcoslat2vordiv(sht_plan *plan, const double *xya_ucos, const double *xya_vcos,
                        int nb, double *wa_vor, double *wa_div);

/* calc_UVCosLat2VorDiv(A, B) of the momentum products
 *   A = cos(phi) (x1 q + z1),  B = cos(phi) (x2 q + z2),
 * formed while the grids load: the xy_A, xy_B of HBEBaroc_MOMRHS_VorDivForm
 * (dynamics/hspm_vfvm/HBEBaroc_hspm_vfvm_mod.f90:394-418; q the vorticity,
 * x1, x2 the velocities, z1, z2 every other term), whose -w_AlphaOptr_xy(A, B)
 * and w_AlphaOptr_xy(B, -A) of :430-434 are (-wa_div, wa_vor) here.  Five
 * grids read once instead of A and B written and read.  z1 and z2 are both
 * given or both NULL (products only).  SpmlUtil_mod.f90:342-368 for the
 * transform itself. */
SHT_API int sht_uvcoslat2vordiv_fma(sht_plan *plan, const double *xya_x1, const double *xya_x2,
                            const double *xya_q, const double *xya_z1, const double *xya_z2,
                            int nb, double *wa_vor, double *wa_div);

/* calc_VorDiv2UV: psi = a^2 LaplaInv(Vor), chi = a^2 LaplaInv(Div),
 * U = cos * AlphaOptr(chi, -psi), V = cos * AlphaOptr(psi, chi)
 * (SpmlUtil_mod.f90:316-340, 370-396). */
SHT_API int sht_vordiv2uv(sht_plan *plan, const double *wa_vor, const double *wa_div,
                  int nb, double *xya_u, double *xya_v);

/* w_Lapla_w, w_LaplaInv_w (SpmlUtil_mod.f90:117): -n(n+1) w and its inverse
 * with the n = 0 mode set to zero (HBEBarot_hspm_vfvm_mod.f90:295-298). */
SHT_API int sht_wa_lapla_wa(sht_plan *plan, const double *wa, int nb, double *out);
SHT_API int sht_wa_laplainv_wa(sht_plan *plan, const double *wa, int nb, double *out);

/* Spectral backward-Euler lateral diffusion, in place:
 * wa(l,k) <- filter(l) wa(l,k) / (1 - dt coef(l))
 * (physics/DOGCM_Phys_hspm_vfvm_mod.f90:638-641, 741-742).  filter may be NULL
 * (all ones).  coef and filter have lm entries. */
SHT_API int sht_wa_diffuse(sht_plan *plan, double *wa, int nb, const double *coef, double dt,
                   const double *filter);

/* AvrLonLat_xy / IntLonLat_xy (SpmlUtil_mod.f90:123-124): one value per level;
 * ya_AvrLon_xya / ya_IntLon_xya: out(jm, nb). */
SHT_API int sht_avrlonlat_xya(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_intlonlat_xya(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_ya_avrlon_xya(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_ya_intlon_xya(sht_plan *plan, const double *xya, int nb, double *out);

/* ------------------------------------------- transforms, device arrays */
/* Same operations on device pointers, enqueued on the plan's stream. */
SHT_API int sht_wa_xya_dev(sht_plan *plan, const double *xya, int nb, double *wa);
SHT_API int sht_xya_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_wa_divlambda_xya_dev(sht_plan *plan, const double *xya, int nb, double *wa);
SHT_API int sht_wa_divmu_xya_dev(sht_plan *plan, const double *xya, int nb, double *wa);
SHT_API int sht_xya_gradlambda_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradmu_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradlon_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_xya_gradlat_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya);
SHT_API int sht_wa_alphaoptr_xya_dev(sht_plan *plan, const double *xya_a, const double *xya_b,
                             int nb, double *wa);
SHT_API int sht_xya_alphaoptr_wa_dev(sht_plan *plan, const double *wa_a, const double *wa_b,
                             int nb, double *xya);
SHT_API int sht_wa_alphaoptr_prod_xya_dev(sht_plan *plan, const double *xya_a, const double *xya_b,
                                  const double *xya_q, int nb, double *wa);
SHT_API int sht_xya_hgrad_wa_dev(sht_plan *plan, const double *wa, int nb, double *xya_lon,
                         double *xya_lat);
SHT_API int sht_xya_hgrad_xya_dev(sht_plan *plan, const double *xya, int nb, double *xya_lon,
                          double *xya_lat);
SHT_API int sht_xya_fluxdiv_xya_dev(sht_plan *plan, const double *xya_a, const double *xya_b, int nb,
                            double *xya);
SHT_API int sht_uvcoslat2vordiv_dev(sht_plan *plan, const double *xya_ucos, const double *xya_vcos,
                            int nb, double *wa_vor, double *wa_div);
SHT_API int sht_uvcoslat2vordiv_fma_dev(sht_plan *plan, const double *xya_x1, const double *xya_x2,
                                const double *xya_q, const double *xya_z1, const double *xya_z2,
                                int nb, double *wa_vor, double *wa_div);
SHT_API int sht_vordiv2uv_dev(sht_plan *plan, const double *wa_vor, const double *wa_div,
                      int nb, double *xya_u, double *xya_v);
SHT_API int sht_wa_lapla_wa_dev(sht_plan *plan, const double *wa, int nb, double *out);
SHT_API int sht_wa_laplainv_wa_dev(sht_plan *plan, const double *wa, int nb, double *out);
SHT_API int sht_wa_diffuse_dev(sht_plan *plan, double *wa, int nb, const double *coef, double dt,
                       const double *filter);
SHT_API int sht_avrlonlat_xya_dev(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_intlonlat_xya_dev(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_ya_avrlon_xya_dev(sht_plan *plan, const double *xya, int nb, double *out);
SHT_API int sht_ya_intlon_xya_dev(sht_plan *plan, const double *xya, int nb, double *out);

/* Fused round trip used by the implicit diffusion step
 * (physics/DOGCM_Phys_hspm_vfvm_mod.f90:638-641):
 * xya <- xy_w( filter * w_xy(xya) / (1 - dt coef) ), in place on device
 * arrays.  coef/filter (lm entries, device pointers) may be NULL (plain
 * round trip). */
SHT_API int sht_roundtrip_diffuse_dev(sht_plan *plan, double *xya, int nb, const double *coef,
                              double dt, const double *filter);

/* ------------------------------------------------- arrays with leading dimensions */

/* Analysis (w_xy) and synthesis (xy_w) of haloed or padded arrays, with the
 * precision chosen per call.  The model keeps its fields as xyz(IA, JA, KA)
 * with halos (IHALO = JHALO = 1, util/grid/DOGCM_GaussSpmVFvmGrid_mod.f90:
 * 158-183) and its loops copy the (IS:IE, JS:JE) section in and out of every
 * SpmlUtil call through explicit-shape dummies (SpmlUtil_mod.f90:110, with
 * the per-level loops of HBEBaroc_hspm_vfvm_mod.f90:160-172).  Here the
 * caller passes the section's first point and the array's leading
 * dimensions instead: grid point (i, j) of level k at
 * xya[i + ldi*(j + ldj*k)] (0 <= i < im, 0 <= j < jm, ldi >= im, ldj >= jm),
 * spectral entry l of level k at wa[l + ldw*k] (ldw >= lm).  Points outside
 * the section (halos, padding) are neither read nor written.  mode is
 * SHT_PREC_FP64 or SHT_PREC_SPLIT for this call only, or -1 for the plan's
 * precision.  With ldi = im, ldj = jm, ldw = lm these are sht_wa_xya /
 * sht_xya_wa (and their _dev forms); otherwise the sections move by pitched
 * copies to and from the plan's staging.  The _dev forms take device
 * pointers and run on the plan's stream without a final synchronisation. */
SHT_API int sht_analysis(sht_plan *plan, const double *xya, int ldi, int ldj, int nb,
                         double *wa, int ldw, int mode);
SHT_API int sht_synthesis(sht_plan *plan, const double *wa, int ldw, int nb,
                          double *xya, int ldi, int ldj, int mode);
SHT_API int sht_analysis_dev(sht_plan *plan, const double *xya, int ldi, int ldj, int nb,
                             double *wa, int ldw, int mode);
SHT_API int sht_synthesis_dev(sht_plan *plan, const double *wa, int ldw, int nb,
                              double *xya, int ldi, int ldj, int mode);

/* ------------------------------------------------- analysis without allocation */

/* No counterpart in the reference: this entry point exists for callers that
 * must not allocate device memory while they run.  Examples are a host whose
 * GPU memory is owned by another pool allocator, a time loop that cannot
 * absorb the device-wide synchronisation cudaMalloc/cudaFree may cause, or a
 * policy of no allocation after start-up.  It computes the same result as
 * sht_wa_xya_dev (w_xy / wa_xya on device arrays).  Its intermediate arrays
 * live in one fixed device array of sht_noalloc_scratch_bytes() bytes
 * (32 MiB), held by every GPU that loads the library until exit.  It calls no
 * allocator.  A batch needing more scratch returns SHT_ERR_TOO_LARGE.  All
 * calls share that array, so calls that overlap on the GPU race: order them
 * on one stream.  The first call on a plan looks up the array's address
 * (cudaGetSymbolAddress); on a device's first lookup the driver loads the
 * array's module and reserves the array (CUDA's default lazy loading).  A
 * call with nb = 0 does only that set-up: make it at start-up, before another
 * pool takes the GPU's memory and before any stream capture.  Stage timing
 * (sht_last_timing) does not cover this entry point.  The plan
 * must already exist (sht_init allocates its tables); in split precision,
 * so must its digit tables, which the plan's first split-precision call of an
 * ordinary entry point allocates (until then this returns
 * SHT_ERR_INVALID_ARG). */
SHT_API int sht_wa_xya_dev_noalloc(sht_plan *plan, const double *xya, int nb, double *wa);
SHT_API unsigned long long sht_noalloc_scratch_bytes(void);

/* ------------------------------------------------ multi-instance batches
 * Many independent transform instances in one step.  Each instance has its
 * own plan (grid and truncation), field-level count nb and device arrays
 * wa (lm x nb, SPML layout) and xya (im x jm x nb).  The instances of one
 * plan run as a single column range through the same kernels as a batched
 * call (per-column pointer tables, no gather copies); different plans run side
 * by side on their own streams.  sht_multi_build groups the instances,
 * optionally times the Legendre variants of every plan and keeps the fastest,
 * and captures each step kind once as a CUDA graph that sht_multi_run replays.
 *
 * The reference holds one grid per process (SpmlUtil_mod.f90:146-160), so
 * this has no counterpart there; it is the batched step API of the transform
 * path (ensemble members or several resolutions in one job).
 *
 * Rules: the batch owns its Fourier and spectral workspaces; the plans'
 * tables must outlive it (sht_multi_destroy before sht_final); grid arrays
 * must be 16-byte aligned, and no array may move after sht_multi_build; runs
 * of one batch are ordered on its own stream.  sht_multi_build runs steps on
 * the registered arrays (warm-up and tuning, as a measuring FFT planner does),
 * so fill them after building. */
typedef struct sht_multi_s sht_multi;

#define SHT_MULTI_SYNTHESIS 1  /* xya = xy_w(wa) for every instance */
#define SHT_MULTI_ANALYSIS 2   /* wa = w_xy(xya) for every instance */
#define SHT_MULTI_ROUND_TRIP 3 /* synthesis, then analysis */

#define SHT_MULTI_AUTOTUNE 1    /* build: time the Legendre variants per plan, keep the fastest */
#define SHT_MULTI_ALLOW_SPLIT 2 /* build: the tuner may choose split precision (<= 1e-11 relative) */
#define SHT_MULTI_NO_GRAPH 4    /* build: launch stage by stage instead of replaying a graph */
#define SHT_MULTI_SIDE_BY_SIDE 8 /* build: size every group's persistent grids for a share of the SMs
                                   (in proportion to its tuned time, or its columns untuned) without
                                   timing the alternative; the autotuner otherwise decides */

/* Creates an empty batch on the current device. */
SHT_API int sht_multi_create(sht_multi **multi);
/* Registers one instance; returns its index through instance (may be NULL). */
SHT_API int sht_multi_add(sht_multi *multi, sht_plan *plan, int nb, double *wa, double *xya, int *instance);
/* Groups, sizes workspaces, tunes (flags above) and captures the graphs. */
SHT_API int sht_multi_build(sht_multi *multi, int flags);
/* Enqueues one step (SHT_MULTI_SYNTHESIS / _ANALYSIS / _ROUND_TRIP) on the
 * batch's stream and returns. */
SHT_API int sht_multi_run(sht_multi *multi, int what);
/* Stream the runs are enqueued on (a cudaStream_t as void*; NULL = the
 * legacy default stream).  Until set, runs go to a stream the batch owns.  A
 * replay is ordered after earlier work on that stream. */
SHT_API int sht_multi_set_stream(sht_multi *multi, void *stream);
/* Waits for the batch's stream and reports device-side errors. */
SHT_API int sht_multi_synchronize(sht_multi *multi);
/* Number of plan groups, and per group: columns (total field-levels), the
 * precision and Legendre kernel option in use, and the tuned round-trip time
 * in ms (0 when not tuned).  NULL outputs are skipped. */
SHT_API int sht_multi_groups(const sht_multi *multi, int *ngroups);
SHT_API int sht_multi_group_info(const sht_multi *multi, int group, int *ncol, int *precision,
                                 int *legendre_kernel, float *tuned_ms);
/* The SHT_OPT_LEGENDRE_TILE value the group runs with (the tuner's choice). */
SHT_API int sht_multi_group_tile(const sht_multi *multi, int group, int *legendre_tile);
/* SMs the group's persistent kernels size their grids for, so that the
 * groups run side by side (0: the whole GPU).  With autotuning the build
 * times the batch both ways and keeps the faster. */
SHT_API int sht_multi_group_sms(const sht_multi *multi, int group, int *sms);
/* Kernel launches one sht_multi_run(what) replays. */
SHT_API int sht_multi_kernels(const sht_multi *multi, int what, int *nkernels);
SHT_API int sht_multi_destroy(sht_multi *multi);

/* ------------------------------------------------------------ diagnostics */

/* Device time in milliseconds of the kernels of the last *_dev call, summed
 * per stage (fft, legendre, spectral); NULL entries are skipped.  Timing is
 * recorded only when enabled with sht_set_timing(plan, 1). */
SHT_API int sht_set_timing(sht_plan *plan, int on);
SHT_API int sht_last_timing(const sht_plan *plan, float *ms_fft, float *ms_legendre,
                    float *ms_spectral);

/* Number of kernel launches issued by this library since process start. */
SHT_API long long sht_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* DOGCM_SHT_H */
