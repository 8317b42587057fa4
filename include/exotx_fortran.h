/*
 * exotx_fortran.h -- the reference's transform and radiation routines under
 * their gfortran names, with by-reference arguments and HOST arrays, so that
 * a Fortran model links libexotx.so in place of the subroutines of
 * legmod.f90, fftmod.f90 and gaussmod.f90 and keeps its call sites.
 *
 * The reference's routines are external subroutines with implicit
 * interfaces; their array sizes are compile-time pumamod parameters, not
 * arguments (legmod.f90:10-11, plasimmod.f90:98-116).  Here exotx_legini_
 * stands in for legini (legmod.f90:30): it registers the resolution, the
 * level count, the model's real kind and the filter knobs once, and every
 * later call takes its dimensions from that registration.
 *
 * Arrays are the model's own host arrays in the reference's layouts (sp(2,
 * NCSP), fc(2,NLON/2,NLAT), x(...,NLEV), radiation x(NHOR,NLEV)), of the
 * model's default real kind: 8 bytes under -fdefault-real-8 (the reference's
 * recommended build), 4 bytes in a 4-byte build (real_bytes in
 * exotx_legini_).  A call copies its inputs to the device, computes on the
 * library's stream in the registered precision (EXOTX_FP64, EXOTX_FP32, or
 * EXOTX_MIXED = tensor-core sets; a single Legendre routine runs its FP32
 * kernel under EXOTX_MIXED), converting on the device where that differs from
 * the host kind, copies the outputs back and returns once they are in host
 * memory.  Calls are serialised by a process-wide lock.
 *
 * Errors: the reference's routines have no status argument and stop the
 * program on failure (fftmod.f90:104-111).  These keep the signatures, so a
 * failing call writes a message to stderr and exits the process with status
 * 1 -- unless exotx_stop_on_error_(0) was called, in which case the call
 * returns and exotx_fortran_status_ reports the status.
 */
#ifndef EXOTX_FORTRAN_H
#define EXOTX_FORTRAN_H

#include "exotx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Registration in place of legini (legmod.f90:30-171; knobs plasimmod.f90:
 * 227, 309-317): NLAT, NLEV, host real kind in bytes (4 or 8), precision
 * (exotx_precision), nfilter/ngptfilter/nspvfilter, landhoskn0, filterkappa,
 * nfilterexp, plavor.  Replaces an earlier registration.  *ierr = status. */
void exotx_legini_(const int *nlat, const int *nlev, const int *real_bytes, const int *prec,
                   const int *nfilter, const int *ngptfilter, const int *nspvfilter,
                   const double *landhoskn0, const double *filterkappa, const int *nfilterexp,
                   const double *plavor, int *ierr);
/* Release the registration and its device buffers. */
void exotx_legfree_(void);
/* Status of the last failing call since the previous query (EXOTX_OK if
 * none), then cleared. */
void exotx_fortran_status_(int *ierr);
/* 1 (default): a failing call prints and exits like the reference's stop;
 * 0: it returns and records its status. */
void exotx_stop_on_error_(const int *flag);

/* gaussmod.f90:5 inigau(klat, pz0, pzw): pz0, pzw are real(kind=8) in the
 * reference whatever the default kind; needs no registration */
void inigau_(const int *klat, double *pz0, double *pzw);
/* legmod.f90:230 sp2fc(sp, fc): sp(2,NCSP) -> fc(2,NLON/2,NLAT), m > NTRU zeroed */
void sp2fc_(const void *sp, void *fc);
/* legmod.f90:262 sp2fcdmu(sp, fc): as sp2fc with the d/dmu table */
void sp2fcdmu_(const void *sp, void *fc);
/* legmod.f90:178 fc2sp(fc, sp), symmetric single-CPU branch */
void fc2sp_(const void *fc, void *sp);
/* legmod.f90:312 dv2uv(pd, pz, pu, pv): NLEV levels; pz is left unchanged */
void dv2uv_(const void *pd, const void *pz, void *pu, void *pv);
/* legmod.f90:356 uv2dv(pu, pv, pd, pz): NLEV levels */
void uv2dv_(const void *pu, const void *pv, void *pd, void *pz);
/* legmod.f90:433 qtend(q, qn, uq, vq): NLEV levels */
void qtend_(void *q, const void *qn, const void *uq, const void *vq);
/* legmod.f90:505 mktend(d, t, z, tn, fu, fv, ke, ut, vt): NLEV levels */
void mktend_(void *d, void *t, void *z, const void *tn, const void *fu, const void *fv, const void *ke,
             const void *ut, const void *vt);
/* fftmod.f90:29 gp2fc(a, n, lot): in place, lot rows of length n */
void gp2fc_(void *a, const int *n, const int *lot);
/* fftmod.f90:64 fc2gp(a, n, lot): in place */
void fc2gp_(void *a, const int *n, const int *lot);
/* radmod.f90:927 radstep.  The reference's radstep takes no arguments and
 * works on module arrays; this one takes them explicitly: the radmod
 * scalars in *par (nhor, nlev, nlon of the call) and HOST pointers to the
 * pumamod column arrays in *io (of the registered real kind; real_bytes is
 * 8 if nothing was registered), updated in place as radstep updates them.
 * Runs in FP64 under a registered EXOTX_FP64 (the default), else in FP32. */
void radstep_(const exotx_rad_params *par, const exotx_rad_io *io);

#ifdef __cplusplus
}
#endif
#endif
