/*
 * exo_oracle.h -- FP64 CPU restatement of ExoPlaSim's spectral-transform core
 * (gaussmod, legmod, fftmod, fft991mod, pyfft compositions) and of radmod's
 * per-column radiation pass.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker: the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark may call
 * it; the product (exoplasim_b200, libexotx) never links or calls it.
 *
 * Parity status: no Fortran compiler exists on the build or GPU hosts and the
 * reference ships no golden vectors for these routines, so the restatement is
 * pinned by known-answer properties (Gaussian quadrature identities, exact
 * DFT definitions, spherical-harmonic orthonormality, radiative limits) and by
 * fixtures generated from independent implementations (numpy.fft,
 * scipy.special), not by outputs of the reference itself: "parity unpinned"
 * against the reference binary.
 *
 * Conventions follow the reference exactly:
 *   spectral  sp[2*NCSP]      (re,im) pairs, m-major triangle m=0..NTRU, n=m..NTRU
 *   Fourier   fc[NLAT][NLON]  per latitude NLON/2 complex (re,im) for m=0..NLON/2-1
 *   grid      gp[NLAT][NLON]  same storage as the Fourier rows
 *   tables    q*[NLAT][NCSP]  Fortran q*(NCSP,NLPP) with NLPP = NLAT
 *   columns   x[lev][NHOR]    Fortran x(NHOR,NLEV) (NHOR fastest)
 */
#ifndef EXO_ORACLE_H
#define EXO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- gaussmod.f90 ---------------- */
void oracle_inigau(int klat, double *pz0, double *pzw);

/* ---------------- legmod.f90 ---------------- */
typedef struct {
    int ntru, nlat, nlon, ncsp;
    double *sid, *gwd;            /* [nlat] */
    double *qi, *qj, *qc, *qe, *qm, *qq, *qu, *qv; /* [nlat][ncsp] */
    double *skgpsp, *skspgp;      /* [ntru+1], index n (0-based total wavenumber) */
} oracle_leg;

/* nfilter 0..4 with the namelist knobs of plasimmod.f90:309-317.
 * pyfft_nfs >= 0 selects the pyfft filter exp(-8 (n/NTRU)^8) (pyfft.f90:152-156)
 * for both directions instead. Returns 0 on success. */
int  oracle_legini(oracle_leg *L, int nlat, int nfilter, int ngptfilter,
                   int nspvfilter, double landhoskn0, double filterkappa,
                   int nfilterexp, int pyfft_nfs);
void oracle_legfree(oracle_leg *L);

void oracle_sp2fc(const oracle_leg *L, const double *sp, double *fc);
void oracle_sp2fcdmu(const oracle_leg *L, const double *sp, double *fc);
/* folded != 0: single-CPU symmetric branch (legmod.f90:191-202 vs 203-220) */
void oracle_fc2sp(const oracle_leg *L, const double *fc, double *sp, int folded);
/* pz is restored on exit; plavor subtracted from mode (0,1) real part */
void oracle_dv2uv(const oracle_leg *L, const double *pd, double *pz,
                  double *pu, double *pv, int nlev, double plavor);
void oracle_uv2dv(const oracle_leg *L, const double *pu, const double *pv,
                  double *pd, double *pz, int nlev, int folded);
void oracle_qtend(const oracle_leg *L, double *q, const double *qn,
                  const double *uq, const double *vq, int nlev, int folded);
void oracle_mktend(const oracle_leg *L, double *d, double *t, double *z,
                   const double *tn, const double *fu, const double *fv,
                   const double *ke, const double *ut, const double *vt,
                   int nlev, int folded);

/* ---------------- fftmod.f90 (radix 8/4/3/2, in place) ---------------- */
/* return 0 on success, -1 if n is not one of the allowed lengths */
int oracle_gp2fc(double *a, int n, int lot);
int oracle_fc2gp(double *a, int n, int lot);
/* fft991mod.f90 contract (definition at fft991mod.f90:147-155), n in its list */
int oracle_gp2fc_991(double *a, int n, int lot);
int oracle_fc2gp_991(double *a, int n, int lot);

/* ---------------- radmod.f90 ---------------- */
typedef struct {
    int nlev, nhor, nlon;      /* nlon: longitudes per latitude row (for ndcycle=0, solang) */
    const double *sigma, *sigmah, *dsigma; /* [nlev] */
    /* planet / physical constants (p_earth.f90 defaults) */
    double ga, gascon, acpd, adv;
    /* radmod namelist (radmod.f90:27-100 defaults) */
    double gsol0, gdist2, zsolar1, zsolar2, rcoeff;
    double tswr1, tswr2, tswr3, tpofmt, acllwr, th2oc, clgray;
    double a0o3, a1o3, aco3, bo3, co3, toffo3, o3scale;
    double rcl1[3], rcl2[3], acl2[3];
    int ndcycle, no3, nswrcl, nclouds, nrscat, newrsc, necham, necham6,
        nstartemp, npbroaden, nswr, nlwr, nsol;
    /* solang inputs (declination etc. come from the orbit module) */
    int nfixed, ncstsol, ngenkeplerian;
    double zdecl, zmins, zrtim, rasc, dawn, solclat, solcdec;
    double zcday;               /* fraction of year for mko3 */
} oracle_radpar;

typedef struct {
    const double *sid, *cola;  /* per latitude row [nhor/nlon] */
    /* inputs, reference layout x[lev*nhor + col] */
    const double *dt, *dq, *dcc, *dql;  /* [nlep][nhor] */
    const double *dqco2;                /* [nlev][nhor] */
    const double *dp, *dls, *dicec;     /* [nhor] */
    double *dqo3;                       /* [nlev][nhor] out if no3==1 else in */
    double *gmu0;                       /* [nhor] out if nsol==1 else in */
    double *dalb;                       /* [nhor] in/out */
    double *dsalb;                      /* [nhor][2] in/out (Fortran dsalb(2,NHOR)) */
    /* outputs */
    double *dfu, *dfd, *dftu, *dftd, *dswfl, *dlwfl, *dflux; /* [nlep][nhor] */
    double *dtdt;                       /* [nlev][nhor] in/out */
    double *dtdtswr, *dtdtlwr, *dconv;  /* [nlev][nhor] */
} oracle_radio;

void oracle_radpar_default(oracle_radpar *p, int nlev, int nhor, int nlon,
                           const double *sigma, const double *sigmah,
                           const double *dsigma);
/* radmod.f90:166-376 band split for a blackbody star (lstarfile false) */
void oracle_solarini(double starbbtemp, double minwavel,
                     double *zsolar1, double *zsolar2, double *rcoeff);
void oracle_solang(const oracle_radpar *p, const double *sid, const double *cola,
                   double *gmu0);
void oracle_mko3(const oracle_radpar *p, const double *sid, const double *dt,
                 const double *dp, double *dqo3);
void oracle_radstep(const oracle_radpar *p, oracle_radio *io);
/* the same for columns j0..j1-1 (whole latitude rows when ndcycle == 0) */
void oracle_solang_range(const oracle_radpar *p, const double *sid, const double *cola,
                         double *gmu0, int j0, int j1);
void oracle_mko3_range(const oracle_radpar *p, const double *sid, const double *dt,
                       const double *dp, double *dqo3, int j0, int j1);
void oracle_radstep_range(const oracle_radpar *p, oracle_radio *io, int j0, int j1);

/* ---------------- grid-point step of gridpointa (exo_oracle_gp.c) ---------------- */
typedef struct {
    int nlev, nhor, nlon, nqspec;
    const double *dsigma, *sigmah, *rdsig, *t0, *t01s2, *tkp;  /* [nlev] */
    const double *g, *c;                                       /* [nlev*nlev], column major */
    double akap, rdbrv, adv, psurf, ww;
    const double *dq;                                          /* [nlev][nhor] when nqspec == 0 */
} oracle_gppar;
void oracle_initsi(int nlev, const double *sigmah, const double *dsigma, const double *t0, double akap,
                   double *g, double *c, double *tkp, double *t01s2, double *rdsig);
void oracle_gridpoint(const oracle_gppar *P, const double *gin, double *gout, double *dw, const double *rcsq);

/* ---------------- semi-implicit spectral step (exo_oracle_spec.c) ---------------- */
typedef struct {
    int nlev, ntru, nqspec, nsponge;
    double delt, delt2, pnu, pnu21, plavor, dampsp;
    const double *t0, *dsigma;                            /* [nlev] */
    const double *g, *tau;                                /* [nlev*nlev] column major */
    const double *bm1;                                    /* [(ntru+1)*nlev*nlev], jn = 0 unused */
    const double *damp, *tdisst, *tdissq, *tdissd, *tdissz, *tfrc;   /* [nlev], scaled rates */
    const double *sak;                                    /* [nlev][NRSP] */
} oracle_specpar;
typedef struct {
    double *sdp, *szp, *stp, *sqp, *spp;   /* time level t (updated to t+dt) */
    double *sdm, *szm, *stm, *sqm, *spm;   /* time level t-dt (filtered) */
    double *sdt, *szt, *stt, *sqt, *spt;   /* tendencies */
    const double *sop, *srp;               /* surface geopotential [NRSP], restoration T [nlev][NRSP] */
} oracle_specstate;
void oracle_tau(int L, const double *sigmah, const double *dsigma, const double *rdsig, const double *tkp,
                const double *t01s2, const double *c, double *tau);
void oracle_makebm(int L, int ntru, double delt, const double *t0, const double *dsigma, const double *g,
                   const double *tau, double *bm1);
void oracle_sak(int L, int ntru, const int *ndel, int nhdiff, double *sak);
void oracle_spectrala(const oracle_specpar *P, oracle_specstate *S);
void oracle_spectrald(const oracle_specpar *P, oracle_specstate *S);

/* ---------------- OpenMP drivers (timed CPU baseline) ---------------- */
int  oracle_num_threads(void);
void oracle_inverse_set(const oracle_leg *L, int nlev, const double *spin, double *gpout,
                        double plavor, int use991);
void oracle_forward_set(const oracle_leg *L, int nlev, double *gpin, double *spout, int use991);
void oracle_inverse_set_d(const oracle_leg *L, int nlev, const double *spin, double *gpout,
                          double plavor, int use991);
void oracle_forward_set_d(const oracle_leg *L, int nlev, double *gpin, double *spout, int use991);
void oracle_radstep_par(const oracle_radpar *p, oracle_radio *io);

#ifdef __cplusplus
}
#endif
#endif
