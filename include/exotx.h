/*
 * exotx.h -- C ABI of the B200 spectral-transform core and radiation column
 * pass of ExoPlaSim (libexotx.so).
 *
 * Plain pointers and sizes only.  Array arguments are DEVICE pointers unless
 * a function says otherwise; the caller owns every field array, the library
 * owns the per-resolution tables inside an exotx_plan.  Every function
 * returns an exotx_status; none aborts the process or traps the GPU.
 *
 * Memory layouts are the reference's (Fortran column-major, first index
 * fastest):
 *   spectral  sp(2,NCSP)           re/im pairs, m-major triangle (m=0..NTRU, n=m..NTRU)
 *   Fourier   fc(2,NLON/2,NLAT)    per latitude NLON/2 complex coefficients,
 *                                  the same storage as a grid row gp(NLON,NLAT)
 *   levels    x(...,NLEV)          fields of one kind stacked level by level
 *   columns   x(NHOR,NLEV)         radiation inputs/outputs, NHOR fastest
 * Latitudes run north to south (sid(1) > 0), as inigau returns them.
 *
 * Precision: EXOTX_FP64 arrays are double; EXOTX_FP32 and EXOTX_MIXED arrays
 * are float.  EXOTX_MIXED runs the Legendre contractions on the tensor cores
 * with 3-term BF16 splits of both operands and FP32 accumulation.
 */
#ifndef EXOTX_H
#define EXOTX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    EXOTX_OK = 0,
    EXOTX_BAD_DIM = 1,        /* resolution / level count / size not supported */
    EXOTX_UNSUPPORTED_N = 2,  /* FFT length not factorable by the supported radices */
    EXOTX_BAD_ARG = 3,        /* null pointer, bad enum, misaligned pointer */
    EXOTX_CUDA_ERR = 4,       /* a CUDA runtime call failed */
    EXOTX_NO_MEM = 5,         /* device allocation failed */
    EXOTX_TIMEOUT = 6,        /* a bounded device-side wait gave up */
    EXOTX_NOT_BUILT = 7       /* the requested path is not available in this build */
} exotx_status;

typedef enum { EXOTX_FP64 = 0, EXOTX_FP32 = 1, EXOTX_MIXED = 2 } exotx_precision;

typedef struct exotx_plan_s *exotx_plan;
typedef void *exotx_stream;   /* a cudaStream_t; NULL = legacy default stream */

/* Resolution and the legmod namelist knobs (plasimmod.f90:227, 309-317). */
typedef struct {
    int nlat;            /* NLAT; NLON = 2*NLAT, NTRU = (NLON-1)/3 (plasimmod.f90:100-101) */
    int nfilter;         /* 0 none, 1 Cesaro, 2 exponential, 3 Lander-Hoskins, 4 Riesz-2 */
    int ngptfilter;      /* apply the filter grid->spectral (0/1) */
    int nspvfilter;      /* apply the filter spectral->grid (0/1) */
    double landhoskn0;   /* Lander-Hoskins critical wavenumber */
    double filterkappa;  /* exponential filter strength */
    int nfilterexp;      /* exponential filter exponent */
    int pyfft_nfs;       /* -1: model filters above; 0/1: pyfft's exp(-8(n/NTRU)^8) switch */
    double plavor;       /* planetary vorticity removed from mode (0,1) by dv2uv */
} exotx_grid_desc;

/* Fill *d with the reference defaults for nlat (no filter, plavor = EZ). */
exotx_status exotx_grid_desc_default(int nlat, exotx_grid_desc *d);

/* Plan = device tables for one resolution, built on the GPU in FP64: the
 * Gaussian Newton iteration (replaces inigau, gaussmod.f90:5-40) and the
 * associated-Legendre recurrence with its eight derived tables (replaces
 * legini, legmod.f90:30-171), plus FP32 and BF16-split copies. */
exotx_status exotx_plan_create(const exotx_grid_desc *d, exotx_plan *out);
exotx_status exotx_plan_destroy(exotx_plan p);
exotx_status exotx_plan_dims(exotx_plan p, int *nlat, int *nlon, int *ntru, int *ncsp);
/* HOST copies of sid(NLAT) and gwd(NLAT) (gaussmod.f90:5 outputs) */
exotx_status exotx_plan_gauss(exotx_plan p, double *sid, double *gwd);
/* HOST copy of one FP64 table q?(NCSP,NLAT) in the reference layout;
 * which = 0..7 for qi,qj,qc,qe,qm,qq,qu,qv (legmod.f90:13-20) */
exotx_status exotx_plan_table(exotx_plan p, int which, double *out);

/* Tunables of a plan's tensor-core sets (no counterpart in the reference):
 * the bytes of m-major Fourier intermediate one inverse (forward) launch
 * covers -- instances are grouped up to it, at least one per launch -- so that
 * the intermediate one kernel writes is still in L2 when the next reads it.
 * Default 512 MB each: fewer, larger launches measured faster than L2-sized
 * ones at T127 L20. */
/* EXOTX_TUNE_INV_HALF: 1 lets the inverse kernel run two CTAs per SM, each
 * holding one parity half of a table, where they fit shared memory; 0 (the
 * default: the two measured alike at T127 L20) keeps one CTA per SM with both
 * halves. */
typedef enum { EXOTX_TUNE_CHUNK_INV = 0, EXOTX_TUNE_CHUNK_FWD = 1, EXOTX_TUNE_INV_HALF = 2 } exotx_tune_key;
exotx_status exotx_plan_tune(exotx_plan p, int key, long long value);

/* inigau (gaussmod.f90:5-40) on the device: sid(nlat), gwd(nlat) device arrays */
exotx_status exotx_inigau(int nlat, double *sid, double *gwd, exotx_stream s);

/* ---- Legendre transforms; nlev fields of the same kind, stacked ---- */
/* sp2fc (legmod.f90:230): sp(2,NCSP,nlev) -> fc(2,NLON/2,NLAT,nlev), m>NTRU zeroed */
exotx_status exotx_sp2fc(exotx_plan p, int prec, const void *sp, void *fc, int nlev, exotx_stream s);
/* sp2fcdmu (legmod.f90:262): as sp2fc with the d/dmu table qj */
exotx_status exotx_sp2fcdmu(exotx_plan p, int prec, const void *sp, void *fc, int nlev, exotx_stream s);
/* fc2sp (legmod.f90:178), symmetric single-CPU branch: fc -> sp */
exotx_status exotx_fc2sp(exotx_plan p, int prec, const void *fc, void *sp, int nlev, exotx_stream s);
/* dv2uv (legmod.f90:312): (div, vort) -> (u cos, v cos) Fourier; pz is not modified */
exotx_status exotx_dv2uv(exotx_plan p, int prec, const void *pd, const void *pz,
                         void *pu, void *pv, int nlev, exotx_stream s);
/* uv2dv (legmod.f90:356): (u, v) Fourier -> (div, vort) */
exotx_status exotx_uv2dv(exotx_plan p, int prec, const void *pu, const void *pv,
                         void *pd, void *pz, int nlev, exotx_stream s);
/* mktend (legmod.f90:505): call-site argument order (d,t,z,tn,fu,fv,ke,ut,vt) */
exotx_status exotx_mktend(exotx_plan p, int prec, void *d, void *t, void *z,
                          const void *tn, const void *fu, const void *fv,
                          const void *ke, const void *ut, const void *vt,
                          int nlev, exotx_stream s);
/* qtend (legmod.f90:433): (q, qn, uq, vq) */
exotx_status exotx_qtend(exotx_plan p, int prec, void *q, const void *qn,
                         const void *uq, const void *vq, int nlev, exotx_stream s);

/* ---- real FFTs of lot rows of length n, in place ---- */
/* gp2fc (fftmod.f90:29 / fft991mod.f90:32): grid rows -> (A0,0,A1,B1,...) x 1/n */
exotx_status exotx_gp2fc(int prec, void *a, int n, int lot, exotx_stream s);
/* fc2gp (fftmod.f90:64 / fft991mod.f90:60): inverse, m=0 imaginary slot ignored */
exotx_status exotx_fc2gp(int prec, void *a, int n, int lot, exotx_stream s);
/* 1 if n is a supported FFT length (2^a 3^b 5^c, 4 <= n <= 4096, n even) */
int exotx_fft_supported(int n);

/* ---- per-timestep transform sets (plasim.f90 gridpointa :2396-2486) ----
 * inverse_set: spin(2*NCSP, 4L+1) = sd[L], st[L], sz[L], sq[L], sp
 *   -> gpout(NHOR, 6L+3) = gu[L], gv[L], gt[L], gd[L], gz[L], gq[L], gpj, gpmt, gp
 *   (invlega, i*m Fourier derivative of ln ps, fc2gp of every field)
 * forward_set: gpin(NHOR, 9L+1) = gtn[L], gqn[L], gut[L], gvt[L], guz[L], gvz[L], gke[L], gvpp, guq[L], gvq[L]
 *   -> spout(2*NCSP, 4L+1) = sdf[L], stf[L], szf[L], sqf[L], spf
 *   (gp2fc of every field, fc2sp(gvpp), mktend, qtend); gpin is not modified */
exotx_status exotx_inverse_set(exotx_plan p, int prec, const void *spin, void *gpout,
                               int nlev, exotx_stream s);
exotx_status exotx_forward_set(exotx_plan p, int prec, const void *gpin, void *spout,
                               int nlev, exotx_stream s);
/* The same sets for ninst independent model states of this resolution stored
 * back to back (spin: ninst x (4L+1) x NRSP, gpout: ninst x (6L+3) x NHOR, ...).
 * The reference runs one state per process (plasim.f90 gridpointa); batching
 * makes fields x levels x states the N extent of the tensor-core contractions. */
exotx_status exotx_inverse_set_batch(exotx_plan p, int prec, const void *spin, void *gpout,
                                     int nlev, int ninst, exotx_stream s);
exotx_status exotx_forward_set_batch(exotx_plan p, int prec, const void *gpin, void *spout,
                                     int nlev, int ninst, exotx_stream s);
/* ---- gridpointd transform sets (plasim.f90 gridpointd :3142-3149, :3415-3428) ----
 * inverse_set_d: spin(2*NCSP, 4L+1) = sd[L], st[L], sz[L], sq[L], sp (as inverse_set)
 *   -> gpout(NHOR, 4L+1) = gu[L], gv[L], gt[L], gq[L], gp
 *   (invlegd, legmod.f90:661-677: dv2uv, sp2fc of st, sq and sp; fc2gp of every field)
 * forward_set_d: gpin(NHOR, 4L) = gtdt[L], gudt[L], gvdt[L], gqdt[L]
 *   -> spout(2*NCSP, 4L) = sdf[L], stf[L], szf[L], sqf[L]
 *   (gp2fc of every field, fc2sp of gtdt and gqdt, uv2dv(gudt, gvdt)); gpin is not modified.
 * EXOTX_MIXED runs the tensor-core kernels of the gridpointa sets with these
 * field maps (uv2dv as mktend's d and z with no kinetic-energy term). */
exotx_status exotx_inverse_set_d(exotx_plan p, int prec, const void *spin, void *gpout,
                                 int nlev, exotx_stream s);
exotx_status exotx_forward_set_d(exotx_plan p, int prec, const void *gpin, void *spout,
                                 int nlev, exotx_stream s);
exotx_status exotx_inverse_set_d_batch(exotx_plan p, int prec, const void *spin, void *gpout,
                                       int nlev, int ninst, exotx_stream s);
exotx_status exotx_forward_set_d_batch(exotx_plan p, int prec, const void *gpin, void *spout,
                                       int nlev, int ninst, exotx_stream s);
/* Both sets for ninst states whose arrays are in HOST memory, laid out as for
 * the _batch calls (h_spin -> h_gpout by the inverse set, h_gpin -> h_spout by
 * the forward set; pass both pointers of a half as NULL to skip it).  The
 * states stream through three device slots on the plan's own three streams,
 * so copies in, transforms and copies out of neighbouring groups of states
 * overlap; host memory should be page-locked (cudaHostAlloc) for that.  The
 * work starts after what is queued on s, and s waits for the last copy out:
 * synchronise s before reading the outputs.  This is the drop-in for a host
 * model's gridpointa (plasim.f90:2396-2486), whose arrays live in host memory. */
exotx_status exotx_sets_host(exotx_plan p, int prec, const void *h_spin, void *h_gpout,
                             const void *h_gpin, void *h_spout, int nlev, int ninst,
                             exotx_stream s);
/* exotx_sets_host for FP64 host arrays whatever prec is: the array kind of a
 * model built with -fdefault-real-8 (the reference's recommended build).
 * With EXOTX_FP32 or EXOTX_MIXED the FP64 arrays are copied to the device as
 * they are and converted there (round to nearest) before the transforms, and
 * the results converted back to FP64 before the copy out, so an 8-byte model
 * runs the tensor-core sets without converting on the host. */
exotx_status exotx_sets_host_f64(exotx_plan p, int prec, const double *h_spin, double *h_gpout,
                                 const double *h_gpin, double *h_spout, int nlev, int ninst,
                                 exotx_stream s);
/* Uneven ensembles (no counterpart in the reference, which runs one model
 * state per process): ninst instances with their own nlat (NLON = 2 NLAT) and
 * level count, MIXED precision (float arrays).  Instances of one resolution
 * and level count form a segment (at most 12 segments); each half of the
 * round trip (plasim.f90 gridpointa :2396-2486, as inverse_set/forward_set)
 * is one tensor-core Legendre launch and one FFT launch over every segment.
 * Arrays are packed: instance i's spectral data (4L+1 x NRSP, input of the
 * inverse half and output of the forward half) start at spec_off[i] floats,
 * its forward-half grid input (9L+1 fields) at gin_off[i], its inverse-half
 * grid output (6L+3 fields) at gout_off[i]; totals[3] are the three lengths. */
typedef struct exotx_ensemble_s *exotx_ensemble;
exotx_status exotx_ensemble_create(int ninst, const int *nlat, const int *nlev, exotx_ensemble *out);
exotx_status exotx_ensemble_destroy(exotx_ensemble e);
/* HOST arrays of ninst offsets (each may be NULL) and totals[3] */
exotx_status exotx_ensemble_layout(exotx_ensemble e, long long *spec_off, long long *gin_off,
                                   long long *gout_off, long long *totals);
exotx_status exotx_ensemble_inverse(exotx_ensemble e, const float *spin, float *gpout, exotx_stream s);
exotx_status exotx_ensemble_forward(exotx_ensemble e, const float *gpin, float *spout, exotx_stream s);
/* tile caps of the inverse column tiles (qi/qj and qu/qv jobs), job order
 * (1 = longest first), split products (6 = 3-term BF16 split, 3 = 2-term) */
exotx_status exotx_ensemble_configure(exotx_ensemble e, int nc_qi, int nc_uv, int sorted, int nprod);
/* Autotuner: times every combination of tile caps {64,128} x {32,64}, job
 * order and split products on these inputs (reps round trips each), keeps
 * only those within 1e-6 relative L2 of the 3-term split, and configures the
 * fastest.  choice (HOST, 4 ints, may be NULL) = nc_qi, nc_uv, sorted, nprod;
 * *best_ms (HOST, may be NULL) = its round-trip time.  Synchronises s. */
exotx_status exotx_ensemble_tune(exotx_ensemble e, const float *spin, float *gpout, const float *gpin,
                                 float *spout, int reps, exotx_stream s, int *choice, float *best_ms);
/* forward_set that allocates no device memory.  No counterpart in the
 * reference (which has no device memory to allocate); it exists for callers
 * that cannot call cudaMalloc where they transform -- a host model whose own
 * pool already holds the device memory, or a timestep loop that must not stall
 * on an allocation call.  exotx_forward_set may grow the plan's work buffer and
 * build FFT twiddle tables on first use; this variant keeps both in a fixed
 * array inside the library of EXOTX_STATIC_WORK_BYTES bytes per GPU, held from
 * the library's first use on that GPU until process exit.  It needs
 *   256-rounded (NLON/2 + NLON/2+1) complex twiddles + (9L+1)*NLAT*(NTRU+1) complex
 * of prec's size (FP64: T42 L20 fits, T63 L20 does not; FP32: T63 L20 fits)
 * and returns EXOTX_BAD_DIM, before any work, for sets that need more.
 * prec is EXOTX_FP64 or EXOTX_FP32 (EXOTX_MIXED -> EXOTX_BAD_ARG).  Results
 * equal exotx_forward_set's.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and copies the FFT twiddles
 * into the array, so make that first call before any stream capture.  A later
 * call whose NLON or precision differs from the twiddles the array holds
 * copies them in again from host memory, which may wait for the stream; do
 * that one outside stream capture too.  All calls on a device share the
 * array: calls that overlap on the GPU (different streams or threads without
 * synchronisation between them) race. */
#define EXOTX_STATIC_WORK_BYTES (16u << 20)
exotx_status exotx_forward_set_noalloc(exotx_plan p, int prec, const void *gpin, void *spout,
                                       int nlev, exotx_stream s);
/* ---- raw output records (outmod.f90 writegp :97-134, writesp :140-169) ----
 * One output field = an 8-word int32 header record and a float32 data record,
 * each framed by 4-byte length markers (Fortran unformatted sequential, as
 * gfortran writes it): 48 + 4n bytes for n values.  kind 0 (writegp) converts
 * n grid values to float32; kind 1 (writesp) multiplies spectral real i by
 * spnorm(i) = (-1)^m / sqrt(2) (plasim.f90:1637-1650) and pscale, adds poff to
 * the first, and converts.  head holds the header words as the model sets
 * them (code, level, date, time, dimensions, step, days per year). */
typedef struct {
    int head[8];
    const void *src;      /* DEVICE array of n values of precision prec (FP64 or FP32) */
    long long n;
    int prec, kind, ntru; /* ntru: truncation of a spectral field */
    double pscale, poff;
} exotx_raw_rec;
/* bytes of the records' image (HOST array of nrec descriptors) */
exotx_status exotx_raw_size(const exotx_raw_rec *recs, int nrec, size_t *nbytes);
/* the byte image of the records, in order, into the DEVICE buffer out
 * (exotx_raw_size bytes); copy it to the host and append it to the file */
exotx_status exotx_raw_pack(const exotx_raw_rec *recs, int nrec, void *out, exotx_stream s);

/* Per-kernel device time (diagnostics; no counterpart in the reference).
 * While enabled, launches of these kernels outside stream capture are
 * bracketed by CUDA events on the launching stream.  exotx_kernel_time
 * waits for the recorded events, returns the summed milliseconds and the
 * launch count of one kernel, and clears that kernel's record. */
typedef enum {
    EXOTX_K_TC_FORWARD = 0,   /* tensor-core forward Legendre (fc2sp + mktend + qtend) */
    EXOTX_K_TC_INVERSE = 1,   /* tensor-core inverse Legendre (dv2uv + sp2fc + sp2fcdmu) */
    EXOTX_K_FFT_FORWARD = 2,  /* gp2fc rows */
    EXOTX_K_FFT_INVERSE = 3,  /* fc2gp rows */
    EXOTX_K_LEG_FORWARD = 4,  /* FP64/FP32 forward Legendre */
    EXOTX_K_LEG_INVERSE = 5,  /* FP64/FP32 inverse Legendre */
    EXOTX_K_RADSTEP = 6,      /* radiation column pass */
    EXOTX_K_SURROGATE = 7,    /* radiation surrogate inference */
    EXOTX_K_COUNT = 8
} exotx_kernel_id;
exotx_status exotx_kernel_timing(int enable);
exotx_status exotx_kernel_time(int kernel, double *ms, long long *launches);

/* Error word of the tensor-core and FFT kernels (0 = none; nonzero = a
 * bounded device-side wait gave up), read after synchronising the stream,
 * then reset. */
exotx_status exotx_tc_error(int *code, exotx_stream s);

/* ---- grid-point step of gridpointa (plasim.f90:2441-2455) ----
 * Between the inverse and the forward set: gp = exp(gp), calcgp (:2587-2755:
 * sigma-dot, adiabatic and vertical-advection tendencies, vorticity and
 * divergence flux terms, non-linear geopotential) and the flux products
 * gut = gu gt, gvt = gv gt, gke = gu^2 + gv^2 + gphi, guq = gu gq, gvq = gv gq.
 * The constants are those calcgp reads from pumamod: levels, the reference
 * profile t0 (dimensionless, T0/ct), the semi-implicit matrices of initsi
 * (:1709-1745; g and c column-major, g[i + nlev*j] = g(i+1,j+1)), rdsig
 * (:1564) and the scalings of :1316-1322. */
typedef struct {
    int nlev, nqspec;
    double akap, rdbrv, adv, psurf, ww;
    double dsigma[64], sigmah[64], rdsig[64], t0[64], t01s2[64], tkp[64];
    double g[64 * 64], c[64 * 64];
} exotx_gp_params;
/* Earth defaults for nlev levels (default sigma levels, a 288 K / 6.5 K/km
 * reference profile) with the derived arrays filled */
exotx_status exotx_gp_params_default(int nlev, exotx_gp_params *p);
/* recompute tkp, t01s2, g, c, rdsig from sigmah, dsigma, t0, akap (initsi) */
exotx_status exotx_gp_params_derive(exotx_gp_params *p);
typedef struct exotx_gpconst_s *exotx_gpconst;   /* the constants on the device */
exotx_status exotx_gpconst_create(const exotx_gp_params *p, exotx_gpconst *out);
exotx_status exotx_gpconst_destroy(exotx_gpconst c);
/* ninst states back to back: gin (ninst x (6L+3) x NHOR, the inverse set's
 * output, gp = ln ps) -> gout (ninst x (9L+1) x NHOR, the forward set's
 * input).  dw (ninst x L x NHOR, may be NULL) receives calcgp's vertical
 * velocity diagnostic.  dq (ninst x L x NHOR) is the grid humidity, read only
 * when nqspec = 0.  FP64 or FP32 (EXOTX_MIXED: FP32) arrays; NHOR and the
 * latitudes come from the plan. */
exotx_status exotx_gridpoint(exotx_plan p, exotx_gpconst c, int prec, const void *gin, void *gout,
                             void *dw, const void *dq, int ninst, exotx_stream s);

/* ---- semi-implicit spectral time step (plasim.f90 spectrala :2757-2918,
 * spectrald :3645-3999), one model state, without their diagnostics ----
 * spectrala: the adiabatic step -- divergence at t from the implicit equation
 * (Hoskins and Simmons 1975 eq. 17, the inverse bm1(n) of makebm), surface
 * pressure and temperature tendencies (eqs. 15, 14), the first part of the
 * Robert-Asselin time filter, the leapfrog step, spp(1:2) = 0.
 * spectrald: the diabatic tendencies (the forward gridpointd set's sdt, szt,
 * stt, sqt) added, the implicit restoration (damp, srp), Rayleigh drag (tfrc)
 * and hyperdiffusion (tdiss*, sak) tendencies, no drag or diffusion of the
 * planetary vorticity, the optional top sponge, the second part of the filter.
 * Rates are in the model's time unit 1/Omega, as plasim.f90:1583-1615 scales
 * them; ndel/nhdiff define sak (:1617-1633). */
typedef struct {
    int nlev, nqspec, nsponge, nhdiff;
    double delt, delt2, pnu, pnu21, plavor, dampsp, akap;
    double t0[64], sigmah[64], dsigma[64];
    double damp[64], tdisst[64], tdissq[64], tdissd[64], tdissz[64], tfrc[64];
    int ndel[64];
} exotx_spec_params;
/* Earth defaults: 32 steps per rotation, pnu = 0.1, PlaSim's dissipation
 * time scales and drag, the reference profile of exotx_gp_params_default */
exotx_status exotx_spec_params_default(int nlev, exotx_spec_params *p);
typedef struct exotx_specconst_s *exotx_specconst;
/* the level matrices (initsi), bm1(n) for n = 1..NTRU (makebm) and sak for the
 * plan's truncation, on the device */
exotx_status exotx_specconst_create(exotx_plan p, const exotx_spec_params *sp, exotx_specconst *out);
exotx_status exotx_specconst_destroy(exotx_specconst c);
/* DEVICE arrays [level][NRSP] (sp*: [NRSP]), updated in place */
typedef struct {
    void *sdp, *szp, *stp, *sqp, *spp;   /* time level t, advanced to t + dt */
    void *sdm, *szm, *stm, *sqm, *spm;   /* time level t - dt, filtered */
    void *sdt, *szt, *stt, *sqt, *spt;   /* tendencies (spectrala reads gridpointa's, spectrald gridpointd's) */
    const void *sop;                     /* surface geopotential [NRSP] (spectrala) */
    const void *srp;                     /* restoration temperature [level][NRSP] (spectrald) */
} exotx_spec_state;
exotx_status exotx_spectrala(exotx_specconst c, int prec, const exotx_spec_state *s, exotx_stream st);
exotx_status exotx_spectrald(exotx_specconst c, int prec, const exotx_spec_state *s, exotx_stream st);
/* the same for ninst states (a HOST array of state structs), in one launch per
 * 12 states; results equal ninst single calls' */
exotx_status exotx_spectrala_batch(exotx_specconst c, int prec, const exotx_spec_state *states, int ninst,
                                   exotx_stream st);
exotx_status exotx_spectrald_batch(exotx_specconst c, int prec, const exotx_spec_state *states, int ninst,
                                   exotx_stream st);

/* ---- radiation column pass (radmod.f90 radstep :927-1110) ---- */
typedef struct {
    int nlev, nhor, nlon;                 /* nlon: longitudes per latitude row */
    double ga, gascon, acpd, adv;         /* p_earth.f90:41-58, plasim.f90:1317-1318 */
    double gsol0, gdist2, zsolar1, zsolar2, rcoeff;
    double tswr1, tswr2, tswr3, tpofmt, acllwr, th2oc, clgray;
    double a0o3, a1o3, aco3, bo3, co3, toffo3, o3scale;
    double rcl1[3], rcl2[3], acl2[3];
    int ndcycle, no3, nswrcl, nclouds, nrscat, newrsc, necham, necham6,
        nstartemp, npbroaden, nswr, nlwr, nsol;
    int nfixed, ncstsol, ngenkeplerian;
    double zdecl, zmins, zrtim, rasc, dawn, solclat, solcdec, zcday;
    double sigma[64], sigmah[64], dsigma[64];   /* nlev <= 64 */
} exotx_rad_params;

typedef struct {
    /* per latitude row (nhor/nlon rows) */
    const void *sid, *cola;
    /* inputs, x(NHOR,NLEP) / x(NHOR,NLEV) */
    const void *dt, *dq, *dcc, *dql, *dqco2;
    const void *dp, *dls, *dicec;         /* (NHOR) */
    void *dqo3;                           /* (NHOR,NLEV): written when no3 == 1, else read */
    void *gmu0;                           /* (NHOR): written when nsol == 1, else read */
    void *dalb;                           /* (NHOR) in/out */
    void *dsalb;                          /* (2,NHOR) in/out */
    /* outputs */
    void *dfu, *dfd, *dftu, *dftd, *dswfl, *dlwfl, *dflux;   /* (NHOR,NLEP) */
    void *dtdt;                           /* (NHOR,NLEV) in/out (tendency is added) */
    void *dtdtswr, *dtdtlwr, *dconv;      /* (NHOR,NLEV) */
    /* optional (NHOR,3): zsolar1, zsolar2, rcoeff per column (a star per
     * column, each from exotx_solarini); NULL = the params' scalars */
    const void *zsol;
} exotx_rad_io;

/* ---- learned radiation surrogate (no counterpart in the reference) ----
 * An MLP (nin -> width x nhidden -> nout, SiLU) trained on columns that
 * exotx_radstep computes; it predicts a column's heating-rate profile and
 * its four surface fluxes.  Training runs in FP32 on the library's kernels
 * (exotx_mlp_backward + exotx_mlp_adam); exotx_rad_surrogate runs the
 * network in BF16 on the tensor cores and sends every column with an input
 * outside the training ranges to the plain radstep kernel. */
typedef struct exotx_mlp_s *exotx_mlp;
/* parameters: per layer l, W_l (dout x din, row-major) then b_l (dout) in one
 * flat FP32 device array; max_batch bounds the rows of forward/backward */
exotx_status exotx_mlp_create(int nin, int width, int nhidden, int nout, int max_batch, exotx_mlp *out);
exotx_status exotx_mlp_destroy(exotx_mlp net);
exotx_status exotx_mlp_params(exotx_mlp net, float **params, float **grads, long long *nparams);
exotx_status exotx_mlp_layer(exotx_mlp net, int layer, long long *w_off, long long *b_off, int *din, int *dout);
/* HOST array of 4*nin + 2*nout floats: feature mean, std, min, max; target mean, std */
exotx_status exotx_mlp_set_norm(exotx_mlp net, const float *host_norm);
/* FP32 forward of n normalised rows X (n x nin) -> Y (n x nout, normalised) */
exotx_status exotx_mlp_forward(exotx_mlp net, const float *X, float *Y, int n, exotx_stream s);
/* forward + backward of the mean squared error against T (n x nout): the
 * gradients land in the net's gradient array; *loss (device) += the loss */
exotx_status exotx_mlp_backward(exotx_mlp net, const float *X, const float *T, int n, float *loss,
                                exotx_stream s);
/* the same with the squared error of element (b, o) weighted by W[b * nout + o]
 * (device, n x nout; NULL = all 1): a loss in the units the outputs are judged in */
exotx_status exotx_mlp_backward_weighted(exotx_mlp net, const float *X, const float *T, const float *W, int n,
                                         float *loss, exotx_stream s);
exotx_status exotx_mlp_adam(exotx_mlp net, float lr, float beta1, float beta2, float eps, int step,
                            exotx_stream s);
/* EXOTX_TIMEOUT if a bounded wait of the training GEMMs (tensor cores, FP32-accurate
 * 3-term BF16 splits) gave up since the library was loaded; synchronises s */
exotx_status exotx_mlp_check(exotx_mlp net, exotx_stream s);
/* BF16 tensor-core copy of the current weights (width 256, nin <= 80, nout <= 32) */
exotx_status exotx_mlp_prepare(exotx_mlp net, exotx_stream s);
/* raw features X (nhor x (3L+9)) and targets Y (nhor x (L+4)) of radstep columns:
 * features T(k), T surface, ln q(k<=L), cloud cover(k), ln ps, albedo, gmu0,
 * ln CO2, zsolar1, rcoeff, sin(lat); targets per level the heating rate
 * (K/day) times (ps / 1e5 Pa)(1 + ADV q), then dfd, dfu, dftd, dftu at the surface */
exotx_status exotx_surr_features(const exotx_rad_params *p, int prec, const exotx_rad_io *io, float *X,
                                 exotx_stream s);
exotx_status exotx_surr_targets(const exotx_rad_params *p, int prec, const exotx_rad_io *io, float *Y,
                                exotx_stream s);
/* Surrogate radiation pass (needs nsol = 0: gmu0 is an input).  In-range
 * columns get dtdt += predicted heating and the surface entries of dfd, dfu,
 * dftd, dftu, dswfl, dlwfl; out-of-range columns go through radstep (every
 * output).  *nfallback (HOST, may be NULL; non-NULL synchronises s) receives
 * the number of fallback columns. */
exotx_status exotx_rad_surrogate(exotx_mlp net, const exotx_rad_params *p, int prec,
                                 const exotx_rad_io *io, int *nfallback, exotx_stream s);

/* Reference defaults (radmod.f90:27-100, p_earth.f90, default sigma levels
 * plasim.f90:1554-1564) for nlev levels and nhor columns in rows of nlon. */
exotx_status exotx_rad_params_default(int nlev, int nhor, int nlon, exotx_rad_params *p);
/* solarini band split (radmod.f90:166-376) for a blackbody star */
exotx_status exotx_solarini(double starbbtemp, double minwavel_m,
                            double *zsolar1, double *zsolar2, double *rcoeff);
/* radstep: solang (nsol=1), mko3 (no3=1), swr, lwr, heating rates.  prec is
 * EXOTX_FP64 (double arrays) or EXOTX_FP32 (float arrays). */
exotx_status exotx_radstep(const exotx_rad_params *p, int prec, const exotx_rad_io *io,
                           exotx_stream s);

/* Diagnostic of the tensor-core path (no counterpart in the reference):
 * C(128 x N) = A(128 x K) * B(N x K)^T on one CTA with tcgen05.mma, FP32
 * inputs split into three BF16 terms, nprod in {1,3,6} split products,
 * FP32 accumulation in tensor memory.  Device pointers, row-major, N and K
 * multiples of 16 (N <= 256, K <= 64).  Synchronises the stream. */
exotx_status exotx_tc_selftest(const float *A, const float *B, float *C, int N, int K, int nprod,
                               exotx_stream s);

/* Human-readable text for a status code. */
const char *exotx_status_string(exotx_status st);
/* Number of kernel launches this library issued so far in this process. */
unsigned long long exotx_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
