// radmod.f90 radiation column pass: host entry points and the FP32 kernel.
// The FP64 kernel lives in radiation_fp64.cu, compiled without FMA
// contraction so that every branch test of the reference (several compare
// differences of nearly equal quantities) sees the same rounding.
#include <cmath>
#include <cstring>
#include <algorithm>
#include "radiation_kernel.cuh"

namespace exotx {
exotx_status launch_radstep_fp64(const RadDev &D, int blocks, int warps, size_t smem, cudaStream_t st);

static exotx_status launch_radstep_fp32(const RadDev &D, int blocks, int warps, size_t smem, cudaStream_t st) {
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_radstep<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaEvent_t ev = ktimer_start(EXOTX_K_RADSTEP, st);
    k_radstep<float><<<blocks, warps * 32, smem, st>>>(D);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_RADSTEP, st, ev);
    return EXOTX_OK;
}
}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_rad_params_default(int nlev, int nhor, int nlon, exotx_rad_params *p) {
    if (!p || nlev < 2 || nlev > RAD_MAXLEV || nhor < 1 || nlon < 1) return EXOTX_BAD_ARG;
    memset(p, 0, sizeof(*p));
    p->nlev = nlev; p->nhor = nhor; p->nlon = nlon;
    p->ga = 9.80665; p->gascon = 287.0;
    p->acpd = p->gascon / 0.286;
    p->adv = 1870.0 / p->acpd - 1.0;
    p->gsol0 = 1367.0; p->gdist2 = 1.0;
    p->zsolar1 = 0.517; p->zsolar2 = 0.483; p->rcoeff = 1.0;
    p->tswr1 = 0.077; p->tswr2 = 0.065; p->tswr3 = 0.0055;
    p->tpofmt = 1.0; p->acllwr = 0.1; p->th2oc = 0.024; p->clgray = -1.0;
    p->a0o3 = 0.25; p->a1o3 = 0.11; p->aco3 = 0.08; p->bo3 = 20000.0;
    p->co3 = 5000.0; p->toffo3 = 0.25; p->o3scale = 1.0;
    const double r1[3] = {0.15, 0.30, 0.60}, a2[3] = {0.05, 0.10, 0.20};
    for (int i = 0; i < 3; i++) { p->rcl1[i] = r1[i]; p->rcl2[i] = r1[i]; p->acl2[i] = a2[i]; }
    p->ndcycle = 1; p->no3 = 1; p->nswrcl = 1; p->nclouds = 1; p->nrscat = 1;
    p->newrsc = 0; p->necham = 1; p->necham6 = 0; p->nstartemp = 0;
    p->npbroaden = 1; p->nswr = 1; p->nlwr = 1; p->nsol = 1;
    p->zrtim = (3.14159265359 + 3.14159265359) / 1440.0;
    p->solclat = 1.0; p->solcdec = 1.0;
    // default sigma levels (plasim.f90:1554-1564)
    for (int j = 0; j < nlev; j++) {
        double z = (double)(j + 1) / (double)nlev;
        p->sigmah[j] = 0.75 * z + 1.75 * z * z * z - 1.5 * z * z * z * z;
    }
    p->dsigma[0] = p->sigmah[0];
    for (int j = 1; j < nlev; j++) p->dsigma[j] = p->sigmah[j] - p->sigmah[j - 1];
    p->sigma[0] = 0.5 * p->sigmah[0];
    for (int j = 1; j < nlev; j++) p->sigma[j] = 0.5 * (p->sigmah[j - 1] + p->sigmah[j]);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_solarini(double starbbtemp, double minwavel, double *zsolar1, double *zsolar2,
                                      double *rcoeff) {
    // band split of radmod.f90:166-376 (blackbody star), host FP64, init only
    if (!zsolar1 || !zsolar2 || !rcoeff || starbbtemp <= 0 || minwavel <= 0) return EXOTX_BAD_ARG;
    const double cst = 0.0143877735383;
    static double wv1[1024], wv2[1024];
    double constg = cst / 5772.0, lwmin = log10(minwavel), hinge = log10(7.5e-7);
    double dl1 = (hinge - lwmin) / 1024.0, dl2 = (-4 - hinge) / 1024.0;
    double bb1[1024], bb2[1024], bbg1[1024], bbg2[1024];
    double const2 = cst / starbbtemp;
    for (int k = 0; k < 1024; k++) {
        wv1[k] = pow(10.0, lwmin + k * dl1);
        wv2[k] = pow(10.0, hinge + k * dl2);
        double w1 = pow(1.0e6 * wv1[k], 5), w2 = pow(1.0e6 * wv2[k], 5);
        bbg1[k] = 1.0 / w1 * 1.0 / (exp(constg / wv1[k]) - 1);
        bbg2[k] = 1.0 / w2 * 1.0 / (exp(constg / wv2[k]) - 1);
        bb1[k] = 1.0 / w1 * 1.0 / (exp(const2 / wv1[k]) - 1);
        bb2[k] = 1.0 / w2 * 1.0 / (exp(const2 / wv2[k]) - 1);
    }
    double z1 = 0, z2 = 0, zg1 = 0, zg2 = 0, zc1 = 0, zc2 = 0, zgc1 = 0, zgc2 = 0;
    auto i4 = [](double w) { return pow(w * 1.0e6, 4); };
    for (int k = 0; k < 1023; k++) {
        double d1 = wv1[k + 1] - wv1[k], d2 = wv2[k + 1] - wv2[k];
        z1 += 0.5 * (bb1[k] + bb1[k + 1]) * d1;
        z2 += 0.5 * (bb2[k] + bb2[k + 1]) * d2;
        zg1 += 0.5 * (bbg1[k] + bbg1[k + 1]) * d1;
        zg2 += 0.5 * (bbg2[k] + bbg2[k + 1]) * d2;
        zc1 += 0.5 * (bb1[k] / i4(wv1[k]) + bb1[k + 1] / i4(wv1[k + 1])) * d1;
        zc2 += 0.5 * (bb2[k] / i4(wv2[k]) + bb2[k + 1] / i4(wv2[k + 1])) * d2;
        zgc1 += 0.5 * (bbg1[k] / i4(wv1[k]) + bbg1[k + 1] / i4(wv1[k + 1])) * d1;
        zgc2 += 0.5 * (bbg2[k] / i4(wv2[k]) + bbg2[k + 1] / i4(wv2[k + 1])) * d2;
    }
    double dj = wv2[0] - wv1[1023];
    z1 += 0.5 * (bb1[1023] + bb2[0]) * dj;
    zc1 += 0.5 * (bb1[1023] / i4(wv1[1023]) + bb2[0] / i4(wv2[0])) * dj;
    zg1 += 0.5 * (bbg1[1023] + bbg2[0]) * dj;
    zgc1 += 0.5 * (bbg1[1023] / i4(wv1[1023]) + bbg2[0] / i4(wv2[0])) * dj;
    double zchi = (zgc1 + zgc2) / (zg1 + zg2);
    *rcoeff = (zc1 + zc2) * 0.517 / z1 / zchi;
    *zsolar1 = z1 / (z1 + z2);
    *zsolar2 = 1.0 - *zsolar1;
    return EXOTX_OK;
}

namespace exotx {
// radstep over all columns, or over the device-side list cols[0 .. *ncols)
// (at most maxcols entries); the list's length is read by the kernel
exotx_status radstep_columns(const exotx_rad_params *p, int prec, const exotx_rad_io *io, const int *cols,
                             const int *ncols, int maxcols, cudaStream_t st) {
    if (!p || !io) return EXOTX_BAD_ARG;
    if (p->nlev < 2 || p->nlev > RAD_MAXLEV || p->nhor < 1 || p->nlon < 1) return EXOTX_BAD_DIM;
    if (prec != EXOTX_FP64 && prec != EXOTX_FP32) return EXOTX_BAD_ARG;
    const void *req[] = {io->dt, io->dq, io->dcc, io->dql, io->dqco2, io->dp, io->dls, io->dicec, io->dqo3,
                         io->gmu0, io->dalb, io->dsalb, io->dfu, io->dfd, io->dftu, io->dftd, io->dswfl,
                         io->dlwfl, io->dflux, io->dtdt, io->dtdtswr, io->dtdtlwr, io->dconv};
    for (const void *q : req) if (!q) return EXOTX_BAD_ARG;
    if ((p->nsol == 1 || p->no3 == 1) && (!io->sid || !io->cola)) return EXOTX_BAD_ARG;
    // sid/cola are indexed by latitude row col/nlon, and ndcycle = 0 averages
    // over rows: columns must fill whole rows
    if ((p->nsol == 1 || p->no3 == 1 || p->ndcycle == 0) && (p->nhor % p->nlon) != 0) return EXOTX_BAD_DIM;
    if ((cols == nullptr) != (ncols == nullptr)) return EXOTX_BAD_ARG;
    if (maxcols <= 0) return EXOTX_OK;
    RadDev D;
    D.p = *p;
    D.sid = io->sid; D.cola = io->cola; D.dt = io->dt; D.dq = io->dq; D.dcc = io->dcc; D.dql = io->dql;
    D.dqco2 = io->dqco2; D.dp = io->dp; D.dls = io->dls; D.dicec = io->dicec;
    D.dqo3 = io->dqo3; D.gmu0 = io->gmu0; D.dalb = io->dalb; D.dsalb = io->dsalb;
    D.dfu = io->dfu; D.dfd = io->dfd; D.dftu = io->dftu; D.dftd = io->dftd; D.dswfl = io->dswfl;
    D.dlwfl = io->dlwfl; D.dflux = io->dflux; D.dtdt = io->dtdt; D.dtdtswr = io->dtdtswr;
    D.dtdtlwr = io->dtdtlwr; D.dconv = io->dconv;
    D.zsol = io->zsol; D.cols = cols; D.ncols = ncols;
    int L = p->nlev, E = L + 1;
    size_t elems = (size_t)6 * E + 7 * L + 11 * L + 8 * L + 8 * E + 2 * E + 4 * L + 2 * (E + 1) + (size_t)L * L + L +
                   6 * E + 32;
    size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    // warps per block limited by the column scratch (<= 200 KB of shared memory)
    int warps = (int)((200 * 1024) / (elems * esz));
    warps = warps < 1 ? 1 : (warps > RAD_WARPS ? RAD_WARPS : warps);
    size_t smem = elems * esz * warps;
    int blocks = (maxcols + warps - 1) / warps;
    // a column list is usually short (often empty): one wave of resident blocks
    // strides over it instead of one block per possible entry
    if (cols) {
        static int nsm = 0;
        if (!nsm) {
            int dev = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1)
                nsm = 148;
        }
        const int per_sm = std::max(1, (int)((227 * 1024) / std::max<size_t>(smem, 1)));
        blocks = std::min(blocks, nsm * per_sm);
    }
    if (prec == EXOTX_FP64) return launch_radstep_fp64(D, blocks, warps, smem, st);
    return launch_radstep_fp32(D, blocks, warps, smem, st);
}
}  // namespace exotx

EXOTX_API exotx_status exotx_radstep(const exotx_rad_params *p, int prec, const exotx_rad_io *io,
                                     exotx_stream s) {
    if (!p || !io) return EXOTX_BAD_ARG;
    return radstep_columns(p, prec, io, nullptr, nullptr, p->nhor, (cudaStream_t)s);
}
