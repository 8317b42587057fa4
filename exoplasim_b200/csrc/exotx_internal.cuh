// Internal declarations shared by the libexotx translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include "exotx.h"

#define EXOTX_API extern "C" __attribute__((visibility("default")))

namespace exotx {

// Counts every kernel launch the library issues (reported through
// exotx_launch_count so callers can tell the native path ran).
void note_launch(unsigned n = 1);

inline exotx_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return EXOTX_OK;
    if (e == cudaErrorMemoryAllocation) return EXOTX_NO_MEM;
    return EXOTX_CUDA_ERR;
}

#define EXOTX_CHECK_LAUNCH()                                        \
    do {                                                            \
        ::exotx::note_launch();                                     \
        cudaError_t e_ = cudaGetLastError();                        \
        if (e_ != cudaSuccess) return ::exotx::cuda_status(e_);     \
    } while (0)

#define EXOTX_TRY(expr)                                             \
    do {                                                            \
        exotx_status st_ = (expr);                                  \
        if (st_ != EXOTX_OK) return st_;                            \
    } while (0)

#define EXOTX_CUDA(expr)                                            \
    do {                                                            \
        cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return ::exotx::cuda_status(e_);     \
    } while (0)

// Programmatic dependent launch.  A kernel launched with launch_pdl may start
// while the kernel before it in the stream is still finishing (once every
// block of that kernel has started and called pdl_trigger); before it touches
// any memory that kernel or an earlier one reads or writes it must call
// pdl_wait, which returns once the previous kernel has completed and its
// writes are visible.  Work before pdl_wait may only use constant data (the
// plan's tables and twiddles).  In a kernel launched without the attribute both
// calls do nothing.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, static_cast<Args &&>(args)...);
}

// Real FFT twiddle tables for one length n, owned by a process-wide cache.
struct FftTables {
    int n = 0, h = 0;            // h = n/2 complex points
    int nfac = 0, fac[16] = {};  // radix schedule of h (product = h)
    double *w64 = nullptr;       // e^{-2 pi i k / h}, k < h   (complex, interleaved)
    float *w32 = nullptr;
    double *r64 = nullptr;       // e^{-2 pi i k / n}, k <= h  (complex, interleaved)
    float *r32 = nullptr;
};
// Returns nullptr (and sets *st) if n is unsupported or allocation fails.
const FftTables *fft_tables(int n, exotx_status *st);

// Mixed-precision table copies built on first use (see legendre_tc.cu).
struct TcTables;
// Device slots, streams and events of the host-memory set pipeline (host_sets.cu).
struct HostPipe;
void host_pipe_free(exotx_plan p);

}  // namespace exotx

struct exotx_plan_s {
    exotx_grid_desc desc;
    int nlat, nlon, ntru, ntp1, ncsp, nlath;
    int kmax;                     // max modes per m = ntp1
    int *d_woff = nullptr;        // first mode index of each m, [ntp1+1]
    double *d_sid = nullptr, *d_gwd = nullptr;
    double *d_qref = nullptr;     // 8 tables, reference layout q(NCSP,NLAT) [t][lat][w]
    // inverse tables qi,qj,qu,qv for northern latitudes, [t][w][j] (j fastest)
    double *d_inv64 = nullptr;
    float *d_inv32 = nullptr;
    // forward tables qc,qe,qm,qq for northern latitudes, per m block [t][woff*nlath + j*K + (n-m)]
    double *d_fwd64 = nullptr;
    float *d_fwd32 = nullptr;
    double *d_fs64 = nullptr, *d_fg64 = nullptr;  // skspgp, skgpsp [ntp1]
    float *d_fs32 = nullptr, *d_fg32 = nullptr;
    // work buffer for the forward transform set (Fourier rows of gpin)
    void *d_work = nullptr;
    size_t work_bytes = 0;
    exotx::TcTables *tc = nullptr;
    exotx::HostPipe *hpipe = nullptr;  // device slots and streams of exotx_sets_host
    // bytes of m-major Fourier intermediate one tensor-core launch covers
    // (instances are grouped up to this, at least one): the intermediate is
    // written by one kernel and read by the next, so it should stay in L2
    // 512 MB: up to 21 T127 L20 instances per inverse launch, 14 per forward;
    // fewer, larger launches measured faster than L2-sized ones (T127 L20,
    // 8 instances: 10.2K round trips/s with one launch per half, 9.5K with 80 MB)
    size_t chunk_inv = (size_t)512 << 20, chunk_fwd = (size_t)512 << 20;
    int inv_half_ok = 0;   // the inverse kernel may run two CTAs per SM where they fit
};

namespace exotx {
// table indices inside d_inv* and d_fwd*
enum { INV_QI = 0, INV_QJ = 1, INV_QU = 2, INV_QV = 3 };
enum { FWD_QC = 0, FWD_QE = 1, FWD_QM = 2, FWD_QQ = 3 };

exotx_status ensure_work(exotx_plan p, size_t bytes);

// Fourier-side addressing: complex element (field f, latitude l, wavenumber m)
// at base + f*fs + l*ls + m*ms (complex units); m < mz are produced.
struct FourierLayout {
    long long fs, ls, ms;
    int mz;
};

// op codes
enum { OP_SP2FC = 0, OP_SP2FCDMU = 1, OP_DV2UV = 2, OP_SP2FC_GPMT = 3 };
enum { OP_FC2SP = 0, OP_UV2DV = 1, OP_QTEND = 2, OP_MKTEND = 3 };

// SIMT Legendre launchers (legendre_simt.cu)
template <typename T>
exotx_status leg_inverse_l(exotx_plan p, int op, const T *a, const T *b, T *oa, T *ob, int nlev,
                           long long a_fs, long long b_fs, FourierLayout L, cudaStream_t s);
template <typename T>
exotx_status leg_forward_l(exotx_plan p, int op, const T *const *in, T *const *out, int nlev,
                           FourierLayout L, long long o_fs, cudaStream_t s);

// FFT launchers (fft.cu).  kf = Fourier coefficients read (inverse) or
// written (forward) per row; the rest are zero.  Fourier side addressed as
// row r, wavenumber k at r*f_rs + k*f_ms (complex units).
template <typename T>
exotx_status fft_forward_l(const T *in, T *out, int n, long long lot, int kout, long long f_rs, long long f_ms,
                           cudaStream_t s);
template <typename T>
exotx_status fft_inverse_l(const T *in, T *out, int n, long long lot, int kin, long long f_rs, long long f_ms,
                           cudaStream_t s);
// twiddle tables on the host (w: n/2 complex, r: n/2+1 complex) and a forward
// FFT reading them from caller-provided device memory (no allocation)
template <typename T>
void fft_twiddles_host(int n, T *w, T *r);
template <typename T>
exotx_status fft_forward_tw(const T *in, T *out, int n, long long lot, int kout, long long f_rs, long long f_ms,
                            const T *w, const T *r, cudaStream_t s);

// FFTs of several segments of FP32 rows (lengths 64..512 with specialised
// kernels) in one launch, for uneven ensembles (fft.cu)
constexpr int FFT_ENS_MAXSEG = 12;
struct FftEnsSeg {
    const float *in;
    float *out;
    long long lot, f_rs, f_ms;
    int n, kf;
    int fold_nlat = 0;  // forward: > 0 writes the equator-folded layout for nlat-row fields
};
// forward FFT into the equator-folded m-major layout of the tensor-core forward
// kernel (E = north + south rows, then O = north - south, per field) (fft.cu).
// rowsum (may be null): also the FP64 sum of every grid row, in the order of
// row_sum_fp64 (register-resident lengths only; EXOTX_NOT_BUILT otherwise)
exotx_status fft_forward_fold(const float *in, float *out, int n, int nlat, long long lot, int kf, long long f_ms,
                              double *rowsum, cudaStream_t s);
bool fft_fold_rowsum(int n);   // whether fft_forward_fold forms row sums for grid length n
exotx_status fft_ens(bool fwd, const FftEnsSeg *segs, int nseg, cudaStream_t s);

// element-wise FP64 <-> FP32 conversion of n device reals (fortran_abi.cu)
exotx_status convert_reals(const void *in, size_t in_esz, void *out, size_t out_esz, size_t n, cudaStream_t s);

// radstep over all columns or a device-side column list (radiation.cu)
exotx_status radstep_columns(const exotx_rad_params *p, int prec, const exotx_rad_io *io, const int *cols,
                             const int *ncols, int maxcols, cudaStream_t st);

// per-kernel event timing (ktimer.cu): start returns nullptr when timing is
// off or the stream is capturing; stop records the pair
cudaEvent_t ktimer_start(int kernel, cudaStream_t s);
void ktimer_stop(int kernel, cudaStream_t s, cudaEvent_t e0);

// tensor-core Legendre (legendre_tc.cu)
exotx_status tc_inverse_set(exotx_plan p, const float *spin, float *four, int nlev, cudaStream_t s);
exotx_status tc_forward_set(exotx_plan p, const float *four, float *spout, int nlev, cudaStream_t s);
exotx_status tc_inverse_batch(exotx_plan p, const float *spin, float *gpout, int L, int ninst, cudaStream_t s);
exotx_status tc_forward_batch(exotx_plan p, const float *gpin, float *spout, int L, int ninst, cudaStream_t s);
// the gridpointd sets (plasim.f90:3142-3149, :3415-3428) on the same kernels
exotx_status tc_inverse_batch_d(exotx_plan p, const float *spin, float *gpout, int L, int ninst, cudaStream_t s);
exotx_status tc_forward_batch_d(exotx_plan p, const float *gpin, float *spout, int L, int ninst, cudaStream_t s);
// uneven ensembles: a segment is a run of instances of one resolution and level count
constexpr int TC_MAXSEG = 12;  // segments per tensor-core launch
struct EnsSeg {
    exotx_plan p;
    int L, ninst;
    const float *spin;  // inverse input, (4L+1) x NRSP per instance
    float *spout;       // forward output, (4L+1) x NRSP per instance
    float *W;           // m-major Fourier intermediate of the segment
};
exotx_status tc_ens_jobs(const EnsSeg *segs, int nseg, int dir, int nc_qi_cap, int nc_uv_cap, bool sort,
                         int4 **d_jobs, int *njobs, size_t *smem);
exotx_status tc_ens_run(const EnsSeg *segs, int nseg, int dir, const int4 *d_jobs, int njobs, size_t smem,
                        int nprod, cudaStream_t s);
bool tc_ens_fwd_folded(const EnsSeg *segs, int nseg);
exotx_status tc_ens_n0(const EnsSeg *segs, const float *const *gpin, int nseg, cudaStream_t s);
// FP32-accurate GEMM on the tensor cores (tc_gemm.cu): C = A B (+ bias), A(m,k) = A[m*am + k*ak],
// B(k,n) = B[k*bk + n*bn]; work: tc_sgemm_work(M, N, K) floats (0: none needed)
exotx_status tc_sgemm(int M, int N, int K, const float *A, long long am, long long ak, const float *B, long long bk,
                      long long bn, float *C, long long ldc, const float *bias, float *work, size_t work_elems,
                      cudaStream_t s);
size_t tc_sgemm_work(int M, int N, int K);
exotx_status tc_sgemm_error(int *err, cudaStream_t s);
exotx_status tc_error_reset(cudaStream_t s);
exotx_status tc_error_read(int *err, cudaStream_t s);
// the same for the FFT kernels' bounded waits (fft.cu)
exotx_status fft_error_reset(cudaStream_t s);
exotx_status fft_error_read(int *err, cudaStream_t s);
exotx_status tc_available();
void tc_free(exotx_plan p);
}  // namespace exotx
