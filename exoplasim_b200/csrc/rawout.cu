// PlaSim raw output records built on the device (outmod.f90 writegp :97-134,
// writesp :140-169; spnorm plasim.f90:1637-1650).
//
// The model writes every output field as two Fortran unformatted sequential
// records: an 8-word int32 header and the field as float32.  Each record is
// framed by 4-byte length markers (gfortran's default), so one field of n
// values takes 4+32+4 + 4+4n+4 bytes.  Spectral fields are normalised the
// ECHAM way on the way out: every coefficient of zonal wavenumber m is
// multiplied by (-1)^m / sqrt(2) and by the field's scale, and the offset is
// added to the first coefficient.  Here one launch forms the byte image of
// all records of an output step in device memory -- markers, headers and
// converted data -- so the host copies it out and writes it with one call.
#include <algorithm>
#include <vector>
#include "exotx_internal.cuh"

namespace exotx {

struct RawRecDev {
    int head[8];
    const void *src;
    long long n;         // values
    long long off;       // byte offset of the record pair in the output
    int prec, kind, ntru;
    double pscale, poff;
};

// spnorm of spectral real index i (0-based, re/im pairs, m-major triangle)
__device__ __forceinline__ double raw_spnorm(long long i, int ntru) {
    long long w = i >> 1;  // complex mode index
    int m = 0;
    long long left = ntru + 1;  // modes of this m
    while (w >= left && left > 0) { w -= left; m++; left--; }
    const double r = 1.0 / sqrt(2.0);  // as plasim.f90:1638 evaluates it
    return (m & 1) ? -r : r;
}

__global__ void k_raw_pack(const RawRecDev *__restrict__ recs, int nrec, unsigned char *__restrict__ out) {
    // one block per record; threads stride over the record's words
    const int r = blockIdx.x;
    if (r >= nrec) return;
    const RawRecDev R = recs[r];
    int *o = reinterpret_cast<int *>(out + R.off);
    const int dbytes = (int)(4 * R.n);
    if (threadIdx.x == 0) {
        o[0] = 32;
        for (int i = 0; i < 8; i++) o[1 + i] = R.head[i];
        o[9] = 32;
        o[10] = dbytes;
        o[11 + R.n] = dbytes;
    }
    // in the model's own real kind, as writesp evaluates it: the product
    // pf * spnorm * pscale is rounded into the float32 record, and the offset
    // is then added to that float32 value in the model's kind
    float *d = reinterpret_cast<float *>(o + 11);
    for (long long i = threadIdx.x; i < R.n; i += blockDim.x) {
        float f;
        if (R.prec == EXOTX_FP64) {
            double v = static_cast<const double *>(R.src)[i];
            if (R.kind == 1) v = v * raw_spnorm(i, R.ntru) * R.pscale;
            f = (float)v;
            if (R.kind == 1 && i == 0) f = (float)((double)f + R.poff);
        } else {
            float v = static_cast<const float *>(R.src)[i];
            if (R.kind == 1) v = v * (float)raw_spnorm(i, R.ntru) * (float)R.pscale;
            f = v;
            if (R.kind == 1 && i == 0) f = f + (float)R.poff;
        }
        d[i] = f;
    }
}

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_raw_size(const exotx_raw_rec *recs, int nrec, size_t *nbytes) {
    if ((!recs && nrec > 0) || nrec < 0 || !nbytes) return EXOTX_BAD_ARG;
    size_t b = 0;
    for (int i = 0; i < nrec; i++) {
        if (recs[i].n < 0) return EXOTX_BAD_ARG;
        b += 48 + 4 * (size_t)recs[i].n;
    }
    *nbytes = b;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_raw_pack(const exotx_raw_rec *recs, int nrec, void *out, exotx_stream s) {
    if ((!recs && nrec > 0) || nrec < 0 || !out) return EXOTX_BAD_ARG;
    if (nrec == 0) return EXOTX_OK;
    std::vector<RawRecDev> h(nrec);
    long long off = 0;
    for (int i = 0; i < nrec; i++) {
        const exotx_raw_rec &q = recs[i];
        if (!q.src || q.n < 1 || q.n > (1LL << 28) || (q.prec != EXOTX_FP64 && q.prec != EXOTX_FP32) ||
            (q.kind != 0 && q.kind != 1) || (q.kind == 1 && q.n > (long long)(q.ntru + 1) * (q.ntru + 2)))
            return EXOTX_BAD_ARG;
        RawRecDev &d = h[i];
        for (int k = 0; k < 8; k++) d.head[k] = q.head[k];
        d.src = q.src; d.n = q.n; d.off = off; d.prec = q.prec; d.kind = q.kind; d.ntru = q.ntru;
        d.pscale = q.pscale; d.poff = q.poff;
        off += 48 + 4 * q.n;
    }
    // the descriptors go to a small device array of their own, released in
    // stream order once the launch has read them
    RawRecDev *dd = nullptr;
    EXOTX_CUDA(cudaMallocAsync((void **)&dd, sizeof(RawRecDev) * nrec, (cudaStream_t)s));
    EXOTX_CUDA(cudaMemcpyAsync(dd, h.data(), sizeof(RawRecDev) * nrec, cudaMemcpyHostToDevice, (cudaStream_t)s));
    k_raw_pack<<<nrec, 256, 0, (cudaStream_t)s>>>(dd, nrec, static_cast<unsigned char *>(out));
    cudaError_t e = cudaGetLastError();
    note_launch();
    cudaFreeAsync(dd, (cudaStream_t)s);
    // the pageable descriptor copy has been staged before cudaMemcpyAsync returned
    return cuda_status(e);
}
