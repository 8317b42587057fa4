// Real FFTs of grid rows with the reference's conventions (fftmod.f90,
// fft991mod.f90:147-155):
//   forward  c_k = (1/n) sum_j x_j e^{-2 pi i jk/n},  stored (A0, 0, A1, B1, ...),
//            k < n/2 (the Nyquist term is not stored)
//   inverse  x_j = A0 + 2 sum_{k=1}^{n/2-1} Re(c_k e^{+2 pi i jk/n}), B0 ignored.
// A length-n real row is transformed as a length-h = n/2 complex sequence
// z_j = x_{2j} + i x_{2j+1} with a self-sorting (Stockham) mixed-radix FFT in
// shared memory, plus the usual even/odd split twiddle e^{-2 pi i k/n}.
// One block transforms R rows; loads and stores of the grid side are
// row-contiguous and coalesced.  The Fourier side may be row-major (the
// reference layout) or m-major (the transform sets' intermediate).
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include "exotx_internal.cuh"
#include "tc_prims.cuh"

namespace exotx {

// complex value; every complex array here starts on a multiple of its size
template <typename T> struct __align__(2 * sizeof(T)) cpx { T x, y; };
template <typename T> __device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
    return cpx<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T> __device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return cpx<T>{a.x + b.x, a.y + b.y}; }
template <typename T> __device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return cpx<T>{a.x - b.x, a.y - b.y}; }
// multiply by e^{sign * i pi/2}: sign=-1 -> -i, sign=+1 -> +i
template <typename T, int S> __device__ __forceinline__ cpx<T> rot90(cpx<T> a) {
    return S < 0 ? cpx<T>{a.y, -a.x} : cpx<T>{-a.y, a.x};
}

// R-point DFT in registers, V[q] = sum_r v[r] e^{S 2 pi i rq/R}
template <typename T, int S> __device__ __forceinline__ void dft2(cpx<T> *v) {
    cpx<T> a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <typename T, int S> __device__ __forceinline__ void dft4(cpx<T> *v) {
    cpx<T> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    cpx<T> b0 = cadd(v[1], v[3]), b1 = rot90<T, S>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0); v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1); v[3] = csub(a1, b1);
}
template <typename T, int S> __device__ __forceinline__ void dft8(cpx<T> *v) {
    const T r = (T)0.70710678118654752440084436210484903928;
    cpx<T> e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4<T, S>(e);
    dft4<T, S>(o);
    // twiddles e^{S 2 pi i q/8}, q = 0..3
    cpx<T> t1 = S < 0 ? cpx<T>{r * (o[1].x + o[1].y), r * (o[1].y - o[1].x)}
                      : cpx<T>{r * (o[1].x - o[1].y), r * (o[1].y + o[1].x)};
    cpx<T> t2 = rot90<T, S>(o[2]);
    cpx<T> t3 = S < 0 ? cpx<T>{r * (-o[3].x + o[3].y), r * (-o[3].y - o[3].x)}
                      : cpx<T>{r * (-o[3].x - o[3].y), r * (-o[3].y + o[3].x)};
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);   v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);   v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);   v[7] = csub(e[3], t3);
}
template <typename T, int S> __device__ __forceinline__ void dft3(cpx<T> *v) {
    const T c = (T)-0.5, s = (T)(S * 0.86602540378443864676372317075293618347);
    cpx<T> t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    cpx<T> m0 = v[0];
    cpx<T> a{m0.x + c * t.x, m0.y + c * t.y};
    cpx<T> b{-s * d.y, s * d.x};  // i*s*d
    v[0] = cadd(m0, t);
    v[1] = cadd(a, b);
    v[2] = csub(a, b);
}
template <typename T, int S> __device__ __forceinline__ void dft5(cpx<T> *v) {
    const T c1 = (T)0.30901699437494742410229341718281905886, c2 = (T)-0.80901699437494742410229341718281905886;
    const T s1 = (T)(S * 0.95105651629515357211643933337938214340), s2 = (T)(S * 0.58778525229247312916870595463907276860);
    cpx<T> t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    cpx<T> d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    cpx<T> a1{v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y};
    cpx<T> a2{v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y};
    // i*(s1 d1 + s2 d2) and i*(s2 d1 - s1 d2)
    cpx<T> b1{-(s1 * d1.y + s2 * d2.y), s1 * d1.x + s2 * d2.x};
    cpx<T> b2{-(s2 * d1.y - s1 * d2.y), s2 * d1.x - s1 * d2.x};
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1); v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[3] = csub(a2, b2);
}

template <typename T, int S, int R>
__device__ __forceinline__ void dftR(cpx<T> *v) {
    if (R == 2) dft2<T, S>(v);
    else if (R == 3) dft3<T, S>(v);
    else if (R == 4) dft4<T, S>(v);
    else if (R == 5) dft5<T, S>(v);
    else dft8<T, S>(v);
}

// One Stockham pass over all rows of the block: src -> dst.
template <typename T, int S, int R>
__device__ void stockham_pass(const cpx<T> *src, cpx<T> *dst, int h, int ns, int rows,
                              const cpx<T> *wtab) {
    const int nq = h / R;
    const int tw_step = h / (ns * R);
    for (int it = threadIdx.x; it < rows * nq; it += blockDim.x) {
        const int row = it / nq, t = it - row * nq;
        const cpx<T> *s = src + (size_t)row * h;
        cpx<T> *d = dst + (size_t)row * h;
        const int k = t % ns;
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[t + r * nq];
#pragma unroll
        for (int r = 1; r < R; r++) {
            cpx<T> w = wtab[r * k * tw_step];
            if (S > 0) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
        dftR<T, S, R>(v);
        const int base = (t / ns) * ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) d[base + r * ns] = v[r];
    }
}

template <typename T, int S>
__device__ const cpx<T> *run_fft(cpx<T> *b0, cpx<T> *b1, int h, int rows, const int *fac, int nfac,
                                 const cpx<T> *wtab) {
    cpx<T> *src = b0, *dst = b1;
    int ns = 1;
    for (int f = 0; f < nfac; f++) {
        const int R = fac[f];
        if (R == 8) stockham_pass<T, S, 8>(src, dst, h, ns, rows, wtab);
        else if (R == 4) stockham_pass<T, S, 4>(src, dst, h, ns, rows, wtab);
        else if (R == 2) stockham_pass<T, S, 2>(src, dst, h, ns, rows, wtab);
        else if (R == 3) stockham_pass<T, S, 3>(src, dst, h, ns, rows, wtab);
        else stockham_pass<T, S, 5>(src, dst, h, ns, rows, wtab);
        __syncthreads();
        ns *= R;
        cpx<T> *tmp = src; src = dst; dst = tmp;
    }
    return src;
}

struct FftLaunch {
    int n, h, nfac, fac[16];
    long long lot;
    int rows_per_block;
    int kf;                 // Fourier coefficients read (inverse) / written (forward)
    long long f_rs, f_ms;   // Fourier addressing (complex units): row stride, m stride
};

// gp (grid rows, contiguous)  ->  Fourier side
template <typename T>
__global__ void __launch_bounds__(256) k_rfft_forward(const T *gp, T *fc, FftLaunch L,
                                                       const cpx<T> *__restrict__ wtab,
                                                       const cpx<T> *__restrict__ rtab) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int h = L.h, n = L.n;
    cpx<T> *b0 = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *b1 = b0 + (size_t)L.rows_per_block * h;
    const long long row0 = (long long)blockIdx.x * L.rows_per_block;
    const int rows = (int)min((long long)L.rows_per_block, L.lot - row0);
    T *braw = reinterpret_cast<T *>(b0);
    const T *src = gp + row0 * n;
    for (int i = threadIdx.x; i < rows * n; i += blockDim.x) braw[i] = src[i];
    __syncthreads();
    const cpx<T> *Z = run_fft<T, -1>(b0, b1, h, rows, L.fac, L.nfac, wtab);
    // split: X_k = E_k + W_n^k O_k, E = (Z_k + conj Z_{h-k})/2, O = (Z_k - conj Z_{h-k})/(2i)
    const T scale = (T)1 / (T)n;
    for (int it = threadIdx.x; it < rows * L.kf; it += blockDim.x) {
        const int row = it / L.kf, k = it - row * L.kf;
        const cpx<T> *z = Z + (size_t)row * h;
        T re, im;
        if (k == 0) {
            re = (z[0].x + z[0].y) * scale;
            im = 0;
        } else {
            cpx<T> a = z[k], b = z[h - k];
            cpx<T> E{(T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y)};
            cpx<T> O{(T)0.5 * (a.y + b.y), (T)0.5 * (b.x - a.x)};
            cpx<T> w = rtab[k];
            cpx<T> wo = cmul(w, O);
            re = (E.x + wo.x) * scale;
            im = (E.y + wo.y) * scale;
        }
        const size_t o = 2 * ((row0 + row) * L.f_rs + (long long)k * L.f_ms);
        fc[o] = re;
        fc[o + 1] = im;
    }
}

// Fourier side  ->  gp (grid rows, contiguous).  in and out may alias when
// the Fourier side uses the row layout (each block owns its rows).
template <typename T>
__global__ void __launch_bounds__(256) k_rfft_inverse(const T *fc, T *gp, FftLaunch L,
                                                       const cpx<T> *__restrict__ wtab,
                                                       const cpx<T> *__restrict__ rtab) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int h = L.h, n = L.n;
    cpx<T> *b0 = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *b1 = b0 + (size_t)L.rows_per_block * h;
    const long long row0 = (long long)blockIdx.x * L.rows_per_block;
    const int rows = (int)min((long long)L.rows_per_block, L.lot - row0);
    // stage c_k (k < kf) into b1, zero above
    for (int it = threadIdx.x; it < rows * h; it += blockDim.x) {
        const int row = it / h, k = it - row * h;
        cpx<T> c{0, 0};
        if (k < L.kf) {
            const size_t o = 2 * ((row0 + row) * L.f_rs + (long long)k * L.f_ms);
            c.x = fc[o];
            c.y = (k == 0) ? (T)0 : fc[o + 1];
        }
        b1[(size_t)row * h + k] = c;
    }
    __syncthreads();
    // Z_k = E_k + i O_k with E = C_k + conj C_{h-k}, O = (C_k - conj C_{h-k}) e^{+2 pi i k/n}, C_h = 0
    for (int it = threadIdx.x; it < rows * h; it += blockDim.x) {
        const int row = it / h, k = it - row * h;
        const cpx<T> *c = b1 + (size_t)row * h;
        cpx<T> a = c[k];
        cpx<T> b = (k == 0) ? cpx<T>{0, 0} : c[h - k];
        cpx<T> E{a.x + b.x, a.y - b.y};
        cpx<T> D{a.x - b.x, a.y + b.y};
        cpx<T> w = rtab[k];
        w.y = -w.y;
        cpx<T> O = cmul(D, w);
        b0[(size_t)row * h + k] = cpx<T>{E.x - O.y, E.y + O.x};
    }
    __syncthreads();
    const cpx<T> *z = run_fft<T, +1>(b0, b1, h, rows, L.fac, L.nfac, wtab);
    const T *zr = reinterpret_cast<const T *>(z);
    T *dst = gp + row0 * n;
    for (int i = threadIdx.x; i < rows * n; i += blockDim.x) dst[i] = zr[i];
}

// ------------------------------------------- length-specialised kernels
// For the model's grid lengths the radix schedule, loop trip counts and
// index divisions are compile-time constants and the twiddles live in
// shared memory; one block transforms ROWS rows.
__host__ __device__ constexpr int radix_count(int h) {
    int r = h, k = 0;
    while (r % 8 == 0 && r > 8) { k++; r /= 8; }
    while (r % 4 == 0) { k++; r /= 4; }
    while (r % 2 == 0) { k++; r /= 2; }
    while (r % 3 == 0) { k++; r /= 3; }
    while (r % 5 == 0) { k++; r /= 5; }
    if (r == 8) k++;
    return k;
}
__host__ __device__ constexpr int radix_at(int h, int idx) {
    int r = h, k = 0;
    while (r % 8 == 0 && r > 8) { if (k++ == idx) return 8; r /= 8; }
    while (r % 4 == 0) { if (k++ == idx) return 4; r /= 4; }
    while (r % 2 == 0) { if (k++ == idx) return 2; r /= 2; }
    while (r % 3 == 0) { if (k++ == idx) return 3; r /= 3; }
    while (r % 5 == 0) { if (k++ == idx) return 5; r /= 5; }
    return 8;
}

// Rows in shared memory keep 2 spare complex slots after every 16 elements:
// the passes' strided reads and writes then spread over the banks (about half
// the wavefronts of a dense row), and even indices stay 16-byte aligned for the
// vector copies.  H is a multiple of 16 for every specialised length.
__host__ __device__ constexpr int fpad(int j) { return j + 2 * (j >> 4); }
template <int H> __host__ __device__ constexpr int fpad_row() { return H + 2 * (H / 16); }

template <typename T, int S, int H, int ROWS, int R, int NS>
__device__ __forceinline__ void pass_ct(const cpx<T> *src, cpx<T> *dst, const cpx<T> *tw) {
    constexpr int NQ = H / R, STEP = H / (NS * R), NIT = ROWS * NQ, HP = fpad_row<H>();
    for (int it = threadIdx.x; it < NIT; it += blockDim.x) {
        const int row = it / NQ, t = it - row * NQ, k = t % NS;
        const cpx<T> *s = src + row * HP;
        cpx<T> *d = dst + row * HP;
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[fpad(t + r * NQ)];
        if constexpr (NS > 1) {  // the first pass has unit twiddles only
#pragma unroll
            for (int r = 1; r < R; r++) {
                cpx<T> w = tw[r * k * STEP];
                if (S > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        dftR<T, S, R>(v);
        const int base = (t / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) d[fpad(base + r * NS)] = v[r];
    }
}

template <typename T, int S, int H, int ROWS, int IDX, int NS>
__device__ __forceinline__ const cpx<T> *passes_ct(cpx<T> *src, cpx<T> *dst, const cpx<T> *tw) {
    if constexpr (IDX >= radix_count(H)) {
        return src;
    } else {
        constexpr int R = radix_at(H, IDX);
        pass_ct<T, S, H, ROWS, R, NS>(src, dst, tw);
        __syncthreads();
        return passes_ct<T, S, H, ROWS, IDX + 1, NS * R>(dst, src, tw);
    }
}

// First pass of a forward transform (unit twiddles), reading its inputs straight
// from the grid rows in global memory: consecutive threads take consecutive
// butterflies of a row, so each of the R loads is a contiguous run per row.
template <typename T, int H, int ROWS, int R>
__device__ __forceinline__ void pass_ct_first_global(const cpx<T> *__restrict__ g, int rows, cpx<T> *dst) {
    constexpr int NQ = H / R, NIT = ROWS * NQ, HP = fpad_row<H>();
    for (int it = threadIdx.x; it < NIT; it += blockDim.x) {
        const int row = it / NQ, t = it - row * NQ;
        cpx<T> v[R];
        if (row < rows) {
            const cpx<T> *s = g + (size_t)row * H;
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = s[t + r * NQ];
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = cpx<T>{0, 0};
        }
        dftR<T, -1, R>(v);
        cpx<T> *d = dst + row * HP;
#pragma unroll
        for (int r = 0; r < R; r++) d[fpad(t * R + r)] = v[r];
    }
}

// The same first pass for rows at arbitrary places: row r of the block is grid
// row rowg[r] (in units of rows), or zeros where rowg[r] < 0.
template <typename T, int H, int ROWS, int R>
__device__ __forceinline__ void pass_ct_first_rows(const cpx<T> *__restrict__ g, const long long *rowg,
                                                   cpx<T> *dst) {
    constexpr int NQ = H / R, NIT = ROWS * NQ, HP = fpad_row<H>();
    for (int it = threadIdx.x; it < NIT; it += blockDim.x) {
        const int row = it / NQ, t = it - row * NQ;
        const long long gr = rowg[row];
        cpx<T> v[R];
        if (gr >= 0) {
            const cpx<T> *s = g + gr * H;
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = s[t + r * NQ];
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = cpx<T>{0, 0};
        }
        dftR<T, -1, R>(v);
        cpx<T> *d = dst + row * HP;
#pragma unroll
        for (int r = 0; r < R; r++) d[fpad(t * R + r)] = v[r];
    }
}

// Passes IDX.. of a transform whose last pass writes the rows < rows straight
// to global memory (row-contiguous): in the last pass NS*R = H, so output
// t + r*NS of consecutive threads is a contiguous run.
template <typename T, int S, int H, int ROWS, int IDX, int NS>
__device__ __forceinline__ void passes_ct_to_global(cpx<T> *src, cpx<T> *dst, const cpx<T> *tw, cpx<T> *g,
                                                    int rows) {
    constexpr int R = radix_at(H, IDX);
    if constexpr (IDX + 1 < radix_count(H)) {
        pass_ct<T, S, H, ROWS, R, NS>(src, dst, tw);
        __syncthreads();
        passes_ct_to_global<T, S, H, ROWS, IDX + 1, NS * R>(dst, src, tw, g, rows);
    } else {
        static_assert(NS * R == H, "last pass");
        constexpr int NQ = H / R, NIT = ROWS * NQ, STEP = H / (NS * R), HP = fpad_row<H>();
        for (int it = threadIdx.x; it < NIT; it += blockDim.x) {
            const int row = it / NQ, t = it - row * NQ, k = t % NS;
            if (row >= rows) continue;
            const cpx<T> *s = src + row * HP;
            cpx<T> v[R];
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = s[fpad(t + r * NQ)];
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    cpx<T> w = tw[r * k * STEP];
                    if (S > 0) w.y = -w.y;
                    v[r] = cmul(v[r], w);
                }
            }
            dftR<T, S, R>(v);
            cpx<T> *d = g + (size_t)row * H;
#pragma unroll
            for (int r = 0; r < R; r++) d[t + r * NS] = v[r];
        }
    }
}

template <typename T> struct vec2 { using t = float4; };
template <> struct vec2<double> { using t = double2; };

// block blk of a forward transform of lot rows (the kernels below pass blockIdx.x)
template <typename T, int N, int ROWS>
__device__ __forceinline__ void rfft_fwd_ct_body(const T *gp, T *fc, long long lot, int kf, long long f_rs,
                                                 long long f_ms, const cpx<T> *__restrict__ wtab,
                                                 const cpx<T> *__restrict__ rtab, long long blk) {
    constexpr int H = N / 2, HP = fpad_row<H>();
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<T> *b0 = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *b1 = b0 + ROWS * HP;
    // twiddles are read from global memory (L1-cached); shared memory holds only the rows
    const cpx<T> *tw = wtab, *rt = rtab;
    const long long row0 = blk * ROWS;
    const int rows = (int)min((long long)ROWS, lot - row0);
    pdl_trigger();
    pdl_wait();   // the grid rows may come from the previous kernel
    // the first pass reads the grid rows directly (unit twiddles); the rest run in shared memory
    constexpr int R0 = radix_at(H, 0);
    pass_ct_first_global<T, H, ROWS, R0>(reinterpret_cast<const cpx<T> *>(gp + row0 * N), rows, b1);
    __syncthreads();
    const cpx<T> *Z = passes_ct<T, -1, H, ROWS, 1, R0>(b1, b0, tw);
    const T scale = (T)1 / (T)N;
    // X_k and X_{H-k} from Z_k and Z_{H-k} (k <= H/2), each Z read once; only
    // k < kf are stored.  Rows fastest: consecutive threads write adjacent
    // entries of the m-major side.
    auto fold = [&](cpx<T> a, cpx<T> b, int k) {
        const cpx<T> E{(T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y)};
        const cpx<T> O{(T)0.5 * (a.y + b.y), (T)0.5 * (b.x - a.x)};
        const cpx<T> wo = cmul(rt[k], O);
        return cpx<T>{(E.x + wo.x) * scale, (E.y + wo.y) * scale};
    };
    const int kh = min(H / 2, kf - 1);   // pairs (k, H-k) with k <= kh cover every k < kf
    for (int it = threadIdx.x; it < ROWS * (kh + 1); it += blockDim.x) {
        const int row = it % ROWS, k = it / ROWS, k2 = H - k;
        if (row >= rows) continue;
        const cpx<T> *z = Z + row * HP;
        T *fr = fc + 2 * ((row0 + row) * f_rs);
        const cpx<T> a = z[fpad(k)];
        if (k == 0) {
            *reinterpret_cast<cpx<T> *>(fr) = cpx<T>{(a.x + a.y) * scale, (T)0};
            continue;
        }
        const cpx<T> b = z[fpad(k2)];
        *reinterpret_cast<cpx<T> *>(fr + 2 * (long long)k * f_ms) = fold(a, b, k);
        if (k2 < kf && k2 != k) *reinterpret_cast<cpx<T> *>(fr + 2 * (long long)k2 * f_ms) = fold(b, a, k2);
    }
}

// Forward transform that writes the Fourier side folded about the equator,
// for the tensor-core Legendre kernel: for a field of nlat grid rows (north to
// south) and latitude pair j < nlat/2 it stores E = X(j) + X(nlat-1-j) at row
// field*nlat + j and O = X(j) - X(nlat-1-j) at row field*nlat + nlat/2 + j of
// the m-major side (complex element (row, m) at row + m*f_ms).  A block takes
// ROWS/2 latitude pairs of one field: rows r and r + ROWS/2 are a pair's
// northern and southern rows.  lot is a multiple of nlat.
template <typename T, int N, int ROWS>
__device__ __forceinline__ void rfft_fwd_fold_body(const T *gp, T *fc, int nlat, long long lot, int kf,
                                                   long long f_ms, const cpx<T> *__restrict__ wtab,
                                                   const cpx<T> *__restrict__ rtab, long long blk) {
    constexpr int H = N / 2, HP = fpad_row<H>(), PR = ROWS / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<T> *b0 = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *b1 = b0 + ROWS * HP;
    // twiddles are read from global memory (L1-cached); shared memory holds only the rows
    const cpx<T> *tw = wtab, *rt = rtab;
    __shared__ long long rowg[ROWS];
    const int nlath = nlat / 2, nbpf = (nlath + PR - 1) / PR;
    const long long field = blk / nbpf;
    const int j0 = (int)(blk - field * nbpf) * PR;
    if (threadIdx.x < ROWS) {
        const int r = threadIdx.x, j = j0 + (r % PR);
        const int lat = r < PR ? j : nlat - 1 - j;
        rowg[r] = (j < nlath && field * nlat < lot) ? field * nlat + lat : -1;
    }
    pdl_trigger();
    __syncthreads();
    pdl_wait();   // the grid rows may come from the previous kernel, which may still read the output
    constexpr int R0 = radix_at(H, 0);
    pass_ct_first_rows<T, H, ROWS, R0>(reinterpret_cast<const cpx<T> *>(gp), rowg, b1);
    __syncthreads();
    const cpx<T> *Z = passes_ct<T, -1, H, ROWS, 1, R0>(b1, b0, tw);
    const T scale = (T)1 / (T)N;
    auto fold = [&](cpx<T> a, cpx<T> b, int k) {
        const cpx<T> E{(T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y)};
        const cpx<T> O{(T)0.5 * (a.y + b.y), (T)0.5 * (b.x - a.x)};
        const cpx<T> wo = cmul(rt[k], O);
        return cpx<T>{(E.x + wo.x) * scale, (E.y + wo.y) * scale};
    };
    auto put = [&](long long row, int k, cpx<T> xn, cpx<T> xs) {
        T *fr = fc + 2 * (row + (long long)k * f_ms);
        *reinterpret_cast<cpx<T> *>(fr) = cpx<T>{xn.x + xs.x, xn.y + xs.y};
        *reinterpret_cast<cpx<T> *>(fr + 2 * (long long)nlath) = cpx<T>{xn.x - xs.x, xn.y - xs.y};
    };
    const int kh = min(H / 2, kf - 1);   // pairs (k, H-k) with k <= kh cover every k < kf
    for (int it = threadIdx.x; it < PR * (kh + 1); it += blockDim.x) {
        const int pr = it % PR, k = it / PR, k2 = H - k, j = j0 + pr;
        if (rowg[pr] < 0) continue;
        const long long row = field * nlat + j;     // E row; O is nlath further
        const cpx<T> *zn = Z + pr * HP, *zs = Z + (pr + PR) * HP;
        const cpx<T> an = zn[fpad(k)], as = zs[fpad(k)];
        if (k == 0) {
            put(row, 0, cpx<T>{(an.x + an.y) * scale, (T)0}, cpx<T>{(as.x + as.y) * scale, (T)0});
            continue;
        }
        const cpx<T> bn = zn[fpad(k2)], bs = zs[fpad(k2)];
        put(row, k, fold(an, bn, k), fold(as, bs, k));
        if (k2 < kf && k2 != k) put(row, k2, fold(bn, an, k2), fold(bs, as, k2));
    }
}

template <typename T, int N, int ROWS>
__device__ __forceinline__ void rfft_inv_ct_body(const T *fc, T *gp, long long lot, int kf, long long f_rs,
                                                 long long f_ms, const cpx<T> *__restrict__ wtab,
                                                 const cpx<T> *__restrict__ rtab, long long blk) {
    constexpr int H = N / 2, HP = fpad_row<H>();
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<T> *b0 = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *b1 = b0 + ROWS * HP;
    // twiddles are read from global memory (L1-cached); shared memory holds only the rows
    const cpx<T> *tw = wtab;
    const long long row0 = blk * ROWS;
    const int rows = (int)min((long long)ROWS, lot - row0);
    pdl_trigger();
    pdl_wait();   // the coefficients come from the previous kernel
    // Z_k and Z_{H-k} of the half-length complex transform from c_k and c_{H-k}
    // (c = 0 for k >= kf, and the m = 0 imaginary part ignored), one load of
    // each coefficient; rows fastest, so consecutive threads read adjacent
    // entries of the m-major side
    auto unfold = [](cpx<T> a, cpx<T> b, cpx<T> w) {
        const cpx<T> E{a.x + b.x, a.y - b.y};
        const cpx<T> D{a.x - b.x, a.y + b.y};
        w.y = -w.y;
        const cpx<T> O = cmul(D, w);
        return cpx<T>{E.x - O.y, E.y + O.x};
    };
    for (int it = threadIdx.x; it < ROWS * (H / 2 + 1); it += blockDim.x) {
        const int row = it % ROWS, k = it / ROWS, k2 = H - k;
        cpx<T> a{0, 0}, b{0, 0};
        if (row < rows) {
            const T *fr = fc + 2 * ((row0 + row) * f_rs);
            if (k < kf) {
                a = *reinterpret_cast<const cpx<T> *>(fr + 2 * (long long)k * f_ms);
                if (k == 0) a.y = 0;
            }
            if (k > 0 && k2 < kf) b = *reinterpret_cast<const cpx<T> *>(fr + 2 * (long long)k2 * f_ms);
        }
        b0[row * HP + fpad(k)] = unfold(a, b, rtab[k]);
        if (k > 0 && k2 != k) b0[row * HP + fpad(k2)] = unfold(b, a, rtab[k2]);
    }
    __syncthreads();
    // the last pass writes the grid rows directly
    passes_ct_to_global<T, +1, H, ROWS, 0, 1>(b0, b1, tw, reinterpret_cast<cpx<T> *>(gp + row0 * N), rows);
}

template <typename T, int N, int ROWS>
__global__ void __launch_bounds__(256) k_rfft_fwd_ct(const T *gp, T *fc, long long lot, int kf, long long f_rs,
                                                      long long f_ms, const cpx<T> *__restrict__ wtab,
                                                      const cpx<T> *__restrict__ rtab) {
    rfft_fwd_ct_body<T, N, ROWS>(gp, fc, lot, kf, f_rs, f_ms, wtab, rtab, blockIdx.x);
}
template <typename T, int N, int ROWS>
__global__ void __launch_bounds__(256) k_rfft_inv_ct(const T *fc, T *gp, long long lot, int kf, long long f_rs,
                                                      long long f_ms, const cpx<T> *__restrict__ wtab,
                                                      const cpx<T> *__restrict__ rtab) {
    rfft_inv_ct_body<T, N, ROWS>(fc, gp, lot, kf, f_rs, f_ms, wtab, rtab, blockIdx.x);
}

template <typename T> constexpr int ct_rows(int n) {
    return (sizeof(T) == 4) ? (n <= 256 ? 16 : 8) : (n <= 256 ? 8 : 4);
}

template <typename T, int N, int ROWS>
__global__ void __launch_bounds__(256) k_rfft_fwd_fold(const T *gp, T *fc, int nlat, long long lot, int kf,
                                                        long long f_ms, const cpx<T> *__restrict__ wtab,
                                                        const cpx<T> *__restrict__ rtab) {
    rfft_fwd_fold_body<T, N, ROWS>(gp, fc, nlat, lot, kf, f_ms, wtab, rtab, blockIdx.x);
}

// ------------------------------------------------ register-resident transforms
// For h = P*Q complex points with P | Q, P threads work a row:
//   Z[q + Q m] = sum_t W_P^{t m} W_h^{t q} sum_j z[t + P j] W_Q^{j q}   (W = e^{-2 pi i/.})
// Thread t takes the Q-point DFT of its column z[t + P j] in registers and
// applies W_h^{t q}; one transposition through shared memory then hands it the
// Q/P whole P-point DFTs q = (Q/P) t + i.  The inverse runs the same steps in
// the other order.  A block of NT threads works RB = NT/P rows.  The grid
// rows (contiguous 4n-byte runs) move between global and shared memory as bulk
// (TMA) copies, one per row; the inverse's Fourier coefficients, runs of only
// RB complex values per wavenumber, arrive by plain coalesced loads.  The
// twiddles W_h^{t q} sit in a per-block table, Q contiguous values per t.
__device__ int g_fft_error;   // nonzero: a bounded wait in an FFT kernel gave up

template <int N> struct RfShape { static constexpr int P = 0, Q = 0, NT = 256; };
template <> struct RfShape<384> { static constexpr int P = 8, Q = 24, NT = 128; };
template <int N> constexpr bool rf_len() { return RfShape<N>::P > 0; }
// Shared memory (complex units unless noted), P = 8:
//   region R, reused in turn for the staged grid rows (row stride RG = 8 mod 16:
//   the two rows of a half-warp on different banks), the transposition (a
//   thread's Q values at stride RT with RT/2 odd, so 8 row-mates' 16-byte
//   accesses fall on distinct banks; rows at stride RS = 8 mod 16), the
//   spectra (odd row stride RZ: 16 rows read at one k on distinct banks) and
//   the staged coefficients of the inverse (k-major, stride RC = RB + 2);
//   then the twiddle table tq[t * RT + q] = W_h^{t q}, the split twiddles
//   rt[k] = e^{-2 pi i k/n} (k < h), and the copy barrier.
template <int N> struct RfLayout {
    static constexpr int P = RfShape<N>::P, Q = RfShape<N>::Q, H = N / 2, NT = RfShape<N>::NT, RB = NT / P;
    static constexpr int RT = Q + 2;
    static constexpr int RS = P * RT + ((8 - (P * RT) % 16) + 16) % 16;
    static constexpr int RZ = H + 1;
    static constexpr int RG = H + 8 + ((H + 8) % 16 == 8 ? 0 : 8);
    static constexpr int RC = RB + 2;
    static constexpr int R = RB * (RS > RZ ? (RS > RG ? RS : RG) : (RZ > RG ? RZ : RG));
    static constexpr size_t OFF_TQ = (size_t)R * 8, OFF_RT = OFF_TQ + (size_t)P * RT * 8,
                            OFF_BAR = OFF_RT + (size_t)H * 8, SMEM = OFF_BAR + 16;
    static_assert(P == 8 && Q % P == 0 && Q % 4 == 0 && (RT / 2) % 2 == 1 && RS % 16 == 8 && RG % 16 == 8, "layout");
    static_assert(H * RC <= R, "the staged coefficients fit region R");
    static_assert(RB <= 32 && RB % 4 == 0, "warp 0 issues one row copy per lane");
};

// cos(2 pi a / 24) for an integer a (multiples of 15 degrees)
__host__ __device__ constexpr double cos24(int a) {
    a = ((a % 24) + 24) % 24;
    if (a > 12) a = 24 - a;
    switch (a) {
        case 0: return 1.0;
        case 1: return 0.96592582628906828675;
        case 2: return 0.86602540378443864676;
        case 3: return 0.70710678118654752440;
        case 4: return 0.5;
        case 5: return 0.25881904510252076235;
        case 6: return 0.0;
        case 7: return -0.25881904510252076235;
        case 8: return -0.5;
        case 9: return -0.70710678118654752440;
        case 10: return -0.86602540378443864676;
        case 11: return -0.96592582628906828675;
        default: return -1.0;
    }
}
// v * e^{S 2 pi i a / 24} for a constant a
template <typename T, int S>
__device__ __forceinline__ cpx<T> cmul_w24(cpx<T> v, int a) {
    a %= 24;
    if (a == 0) return v;
    if (a == 6) return rot90<T, S>(v);
    if (a == 12) return cpx<T>{-v.x, -v.y};
    if (a == 18) return rot90<T, -S>(v);
    const T c = (T)cos24(a), s = (T)(S * cos24(a - 6));   // sin(x) = cos(x - pi/2)
    return cpx<T>{v.x * c - v.y * s, v.x * s + v.y * c};
}
// 24-point DFT in registers, V[k] = sum_n v[n] e^{S 2 pi i nk/24}:
// n = 8 n1 + n2, k = k1 + 3 k2; 3-point DFTs over n1, twiddles W_24^{n2 k1},
// 8-point DFTs over n2
template <typename T, int S>
__device__ __forceinline__ void dft24(cpx<T> *v) {
    cpx<T> a[24];
#pragma unroll
    for (int n2 = 0; n2 < 8; n2++) {
        cpx<T> t[3] = {v[n2], v[8 + n2], v[16 + n2]};
        dft3<T, S>(t);
#pragma unroll
        for (int k1 = 0; k1 < 3; k1++) a[3 * n2 + k1] = cmul_w24<T, S>(t[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        cpx<T> t[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; n2++) t[n2] = a[3 * n2 + k1];
        dft8<T, S>(t);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) v[k1 + 3 * k2] = t[k2];
    }
}
template <typename T, int S, int Q>
__device__ __forceinline__ void dftQ(cpx<T> *v) {
    static_assert(Q == 24, "register DFT length");
    dft24<T, S>(v);
}

// bulk copy shared -> global in this thread's bulk group (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_s2g(void *dst_gmem, const void *src_smem, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
                 "r"(tc::smem_u32(src_smem)), "r"(bytes)
                 : "memory");
}
// returns once this thread's bulk stores have read their shared-memory sources
__device__ __forceinline__ void bulk_commit_wait_read() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

template <int N>
struct RfSmem {
    using Lay = RfLayout<N>;
    cpx<float> *r, *tq, *rt;
    uint64_t *bar;
    __device__ explicit RfSmem(unsigned char *raw)
        : r(reinterpret_cast<cpx<float> *>(raw)), tq(reinterpret_cast<cpx<float> *>(raw + Lay::OFF_TQ)),
          rt(reinterpret_cast<cpx<float> *>(raw + Lay::OFF_RT)), bar(reinterpret_cast<uint64_t *>(raw + Lay::OFF_BAR)) {}
};

// Block set-up from constant data only (runs before the dependent-launch wait):
// the copy barrier and the per-block twiddle tables.  Ends with a block barrier.
template <int N>
__device__ __forceinline__ void rf_setup(const RfSmem<N> &S, const cpx<float> *__restrict__ w,
                                         const cpx<float> *__restrict__ rt) {
    using Lay = RfLayout<N>;
    if (threadIdx.x == 0) {
        tc::mbar_init(S.bar, 1);
        tc::mbar_fence_init();
    }
    for (int i = threadIdx.x; i < Lay::P * Lay::Q; i += blockDim.x) {
        const int t = i / Lay::Q, q = i - t * Lay::Q;
        S.tq[t * Lay::RT + q] = w[t * q];   // t q < h
    }
    for (int k = threadIdx.x; k < Lay::H; k += blockDim.x) S.rt[k] = rt[k];
    __syncthreads();
}

// Waits for the block's bulk loads; false (block-uniform, error word set) if the bounded wait gave up.
// After a timeout every thread waits once more (bounded) for copies still in
// flight, so none lands in shared memory after the block has left (out of
// line: the error path takes no registers from the transform).
__device__ __noinline__ void rf_loads_timed_out(uint64_t *bar, uint32_t phase) {
    if (threadIdx.x == 0) atomicExch(&g_fft_error, 1);
    tc::mbar_wait(bar, phase);
}
__device__ __forceinline__ bool rf_wait_loads(uint64_t *bar, uint32_t phase = 0) {
    const bool ok = __syncthreads_and(tc::mbar_wait(bar, phase)) != 0;
    if (!ok) rf_loads_timed_out(bar, phase);
    return ok;
}

// FP64 sum of a grid row of 2 P Q reals held by P consecutive lanes, lane t
// holding the complex elements t + P j (j < Q): each lane adds its values in
// j order (real part first), then the P lanes combine by an xor butterfly, so
// every lane ends with the same value.  The n = 0 kernel (legendre_tc.cu) reproduces
// this order when it sums the rows from global memory.
template <int P, int Q>
__device__ __forceinline__ double row_sum_fp64(const cpx<float> *v) {
    double a = 0.0;
#pragma unroll
    for (int j = 0; j < Q; j++) {
        a += (double)v[j].x;
        a += (double)v[j].y;
    }
#pragma unroll
    for (int o = 1; o < P; o <<= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}

// Warp 0 issues one bulk copy per row of the block into `stage` (row stride
// RG), completing on `bar`; rows without a source (grow(r) < 0) are zeroed by
// their own threads.  grow(r) is row r's index in g (rows of n floats).
template <int N, typename RowOf>
__device__ __forceinline__ void rf_issue_rows(const float *__restrict__ g, RowOf grow, cpx<float> *stage,
                                              uint64_t *bar) {
    using Lay = RfLayout<N>;
    constexpr int P = Lay::P, H = Lay::H, RB = Lay::RB;
    const int t = threadIdx.x % P, r = threadIdx.x / P;
    if (threadIdx.x < 32) {
        const long long gr = threadIdx.x < RB ? grow(threadIdx.x) : -1ll;
        const unsigned valid = __ballot_sync(0xffffffffu, gr >= 0);
        if (threadIdx.x == 0) tc::mbar_arrive_expect_tx(bar, (uint32_t)__popc(valid) * (uint32_t)(N * 4));
        __syncwarp();
        if (gr >= 0) tc::bulk_g2s(stage + threadIdx.x * Lay::RG, g + gr * N, N * 4, bar);
    }
    if (grow(r) < 0) {   // zero rows: written here, never by a copy
        for (int j = t; j < H; j += P) stage[r * Lay::RG + j] = cpx<float>{0.f, 0.f};
    }
}

// Forward complex transform of the block's RB rows staged in `stage` (the
// loads complete); afterwards row r's Z[k] sits at x[r * RZ + k] (visible to
// the block).  `stage` and `x` may be the same region.  after_read() runs
// once every thread has its row values in registers (a block barrier lies
// before it), before x is written.
template <int N, bool RSUM = false, int RZ = RfLayout<N>::RZ, typename AfterRead>
__device__ __forceinline__ void rf_forward_core(const cpx<float> *stage, cpx<float> *x, const cpx<float> *tqs,
                                                AfterRead after_read, double *rsum = nullptr) {
    using Lay = RfLayout<N>;
    constexpr int P = Lay::P, Q = Lay::Q, QP = Q / P;
    const int t = threadIdx.x % P, r = threadIdx.x / P;
    cpx<float> v[Q];
    const cpx<float> *s = stage + r * Lay::RG + t;
#pragma unroll
    for (int j = 0; j < Q; j++) v[j] = s[P * j];
    __syncthreads();   // the staged rows are read
    after_read();
    if constexpr (RSUM) *rsum = row_sum_fp64<P, Q>(v);   // after the next loads are on their way
    dftQ<float, -1, Q>(v);
    const cpx<float> *tq = tqs + t * Lay::RT;
#pragma unroll
    for (int q = 2; q < Q; q += 2) {
        const float4 f = *reinterpret_cast<const float4 *>(tq + q);
        v[q] = cmul(v[q], cpx<float>{f.x, f.y});
        v[q + 1] = cmul(v[q + 1], cpx<float>{f.z, f.w});
    }
    v[1] = cmul(v[1], tq[1]);
    cpx<float> *xr = x + r * Lay::RS;
#pragma unroll
    for (int q = 0; q < Q; q += 2)
        *reinterpret_cast<float4 *>(xr + t * Lay::RT + q) = make_float4(v[q].x, v[q].y, v[q + 1].x, v[q + 1].y);
    __syncthreads();
    cpx<float> z[QP][P];
#pragma unroll
    for (int i = 0; i < QP; i++) {
#pragma unroll
        for (int u = 0; u < P; u++) z[i][u] = xr[u * Lay::RT + QP * t + i];
        dft8<float, -1>(z[i]);
    }
    __syncthreads();   // the spectra overwrite the transposition buffer
    cpx<float> *zs = x + r * RZ;
#pragma unroll
    for (int i = 0; i < QP; i++)
#pragma unroll
        for (int m = 0; m < P; m++) zs[QP * t + i + Q * m] = z[i][m];
    __syncthreads();
}

// Forward complex transform of the block's RB rows; afterwards row r's Z[k]
// sits at S.r[r * RZ + k] (visible to the block).  grow(r) is row r's index in
// g (rows of n floats), or < 0 for a zero row.  False if the loads timed out.
template <int N, typename RowOf>
__device__ __forceinline__ bool rf_forward_rows(const float *__restrict__ g, RowOf grow, const RfSmem<N> &S) {
    rf_issue_rows<N>(g, grow, S.r, S.bar);
    if (!rf_wait_loads(S.bar)) return false;
    rf_forward_core<N>(S.r, S.r, S.tq, [] {});
    return true;
}

// the Fourier coefficient X_k of a real row from Z_k and Z_{h-k} of its
// half-length complex transform (k > 0), scaled by 1/n
__device__ __forceinline__ cpx<float> rf_split(cpx<float> a, cpx<float> b, cpx<float> wk, float scale) {
    const cpx<float> E{0.5f * (a.x + b.x), 0.5f * (a.y - b.y)};
    const cpx<float> O{0.5f * (a.y + b.y), 0.5f * (b.x - a.x)};
    const cpx<float> wo = cmul(wk, O);
    return cpx<float>{(E.x + wo.x) * scale, (E.y + wo.y) * scale};
}

// rfft_fwd_ct_body for the register-resident lengths: RB rows per block
template <int N>
__device__ __forceinline__ void rfft_fwd_rf_body(const float *gp, float *fc, long long lot, int kf, long long f_rs,
                                                 long long f_ms, const cpx<float> *__restrict__ w,
                                                 const cpx<float> *__restrict__ rt, long long blk) {
    using Lay = RfLayout<N>;
    constexpr int H = Lay::H, RB = Lay::RB;
    extern __shared__ __align__(16) unsigned char smraw[];
    const RfSmem<N> S(smraw);
    const long long row0 = blk * RB;
    const int rows = (int)min((long long)RB, lot - row0);
    pdl_trigger();
    rf_setup<N>(S, w, rt);
    pdl_wait();   // the grid rows may come from the previous kernel
    if (!rf_forward_rows<N>(gp, [&](int r) { return r < rows ? row0 + r : -1ll; }, S)) return;
    const float scale = 1.f / (float)N;
    const int kh = min(H / 2, kf - 1);   // pairs (k, h-k) with k <= kh cover every k < kf
    const bool kfast = f_ms == 1;        // row-major Fourier side: k fastest across threads
    for (int it = threadIdx.x; it < RB * (kh + 1); it += blockDim.x) {
        const int r = kfast ? it / (kh + 1) : it % RB, k = kfast ? it - r * (kh + 1) : it / RB, k2 = H - k;
        if (r >= rows) continue;
        const cpx<float> *z = S.r + r * Lay::RZ;
        cpx<float> *fr = reinterpret_cast<cpx<float> *>(fc) + (row0 + r) * f_rs;
        const cpx<float> a = z[k];
        if (k == 0) {
            fr[0] = cpx<float>{(a.x + a.y) * scale, 0.f};
            continue;
        }
        const cpx<float> b = z[k2];
        fr[(long long)k * f_ms] = rf_split(a, b, S.rt[k], scale);
        if (k2 < kf && k2 != k) fr[(long long)k2 * f_ms] = rf_split(b, a, S.rt[k2], scale);
    }
}

// rfft_fwd_fold_body for the register-resident lengths: a block takes RB/2
// latitude pairs of one field, rows r and r + RB/2 being a pair's northern and
// southern rows
template <int N>
__device__ __forceinline__ void rfft_fwd_fold_rf_body(const float *gp, float *fc, int nlat, long long lot, int kf,
                                                      long long f_ms, const cpx<float> *__restrict__ w,
                                                      const cpx<float> *__restrict__ rt, long long blk) {
    using Lay = RfLayout<N>;
    constexpr int H = Lay::H, RB = Lay::RB, PR = RB / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    const RfSmem<N> S(smraw);
    const int nlath = nlat / 2, nbpf = (nlath + PR - 1) / PR;
    const long long field = blk / nbpf;
    const int j0 = (int)(blk - field * nbpf) * PR;
    const bool fin = field * nlat < lot;
    pdl_trigger();
    rf_setup<N>(S, w, rt);
    pdl_wait();   // the grid rows may come from the previous kernel, which may still read the output
    auto grow = [&](int r) {
        const int j = j0 + (r % PR);
        return (fin && j < nlath) ? field * nlat + (r < PR ? j : nlat - 1 - j) : -1ll;
    };
    if (!rf_forward_rows<N>(gp, grow, S)) return;
    const float scale = 1.f / (float)N;
    auto put = [&](long long row, int k, cpx<float> xn, cpx<float> xs) {
        cpx<float> *fr = reinterpret_cast<cpx<float> *>(fc) + row + (long long)k * f_ms;
        fr[0] = cpx<float>{xn.x + xs.x, xn.y + xs.y};
        fr[nlath] = cpx<float>{xn.x - xs.x, xn.y - xs.y};
    };
    const int kh = min(H / 2, kf - 1);
    for (int it = threadIdx.x; it < PR * (kh + 1); it += blockDim.x) {
        const int pr = it % PR, k = it / PR, k2 = H - k, j = j0 + pr;
        if (!fin || j >= nlath) continue;
        const long long row = field * nlat + j;     // E row; O is nlath further
        const cpx<float> *zn = S.r + pr * Lay::RZ, *zs = S.r + (pr + PR) * Lay::RZ;
        const cpx<float> an = zn[k], as = zs[k];
        if (k == 0) {
            put(row, 0, cpx<float>{(an.x + an.y) * scale, 0.f}, cpx<float>{(as.x + as.y) * scale, 0.f});
            continue;
        }
        const cpx<float> bn = zn[k2], bs = zs[k2], wk = S.rt[k];
        put(row, k, rf_split(an, bn, wk, scale), rf_split(as, bs, wk, scale));
        if (k2 < kf && k2 != k) {
            const cpx<float> wk2 = S.rt[k2];
            put(row, k2, rf_split(bn, an, wk2, scale), rf_split(bs, as, wk2, scale));
        }
    }
}

// Persistent form of rfft_fwd_fold_rf_body.  A block sets up its twiddle
// tables once and walks the items blk = blockIdx.x, + gridDim.x, ... (an item
// is RB/2 latitude pairs of one field).  The grid rows are staged in their own
// region G, apart from the transposition/spectra region X, so the bulk loads
// of the next item are issued as soon as this item's rows are in registers
// and arrive while it is transformed and written out.
template <int N> struct RfPLayout {
    using Lay = RfLayout<N>;
    // spectra row stride of the folded kernel: RZF = 2 mod 16, so a half-warp's
    // eight latitude pairs at two consecutive k fall on 16 distinct bank pairs
    static constexpr int RZF = Lay::H + 2;
    static_assert(RZF % 16 == 2, "spectra stride");
    static constexpr int RX = Lay::RS > RZF ? Lay::RS : RZF;
    static constexpr size_t OFF_X = (size_t)Lay::RB * Lay::RG * 8, OFF_TQ = OFF_X + (size_t)Lay::RB * RX * 8,
                            OFF_RT = OFF_TQ + (size_t)Lay::P * Lay::RT * 8, OFF_BAR = OFF_RT + (size_t)Lay::H * 8,
                            SMEM = OFF_BAR + 16;
    static_assert(OFF_X % 16 == 0 && OFF_TQ % 16 == 0 && OFF_BAR % 16 == 0, "16-byte aligned regions");
};

template <int N, bool RSUM>
__global__ void __launch_bounds__(128) k_rfft_fwd_fold_rf_p(const float *gp, float *fc, int nlat, long long lot,
                                                             int kf, long long f_ms, long long nitems,
                                                             const cpx<float> *__restrict__ w,
                                                             const cpx<float> *__restrict__ rt, double *rowsum) {
    using Lay = RfLayout<N>;
    using PL = RfPLayout<N>;
    constexpr int H = Lay::H, RB = Lay::RB, PR = RB / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<float> *G = reinterpret_cast<cpx<float> *>(smraw), *X = reinterpret_cast<cpx<float> *>(smraw + PL::OFF_X);
    cpx<float> *tqs = reinterpret_cast<cpx<float> *>(smraw + PL::OFF_TQ);
    cpx<float> *rts = reinterpret_cast<cpx<float> *>(smraw + PL::OFF_RT);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + PL::OFF_BAR);
    const int nlath = nlat / 2, nbpf = (nlath + PR - 1) / PR;
    pdl_trigger();
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_fence_init();
    }
    for (int i = threadIdx.x; i < Lay::P * Lay::Q; i += blockDim.x) {
        const int t = i / Lay::Q, q = i - t * Lay::Q;
        tqs[t * Lay::RT + q] = w[t * q];   // t q < h
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) rts[k] = rt[k];
    __syncthreads();
    pdl_wait();   // the grid rows may come from the previous kernel, which may still read the output
    auto grow_of = [&](long long item) {
        const long long field = item / nbpf;
        const int j0 = (int)(item - field * nbpf) * PR;
        const bool fin = field * nlat < lot;
        return [=](int r) {
            const int j = j0 + (r % PR);
            return (fin && j < nlath) ? field * nlat + (r < PR ? j : nlat - 1 - j) : -1ll;
        };
    };
    long long item = blockIdx.x;
    if (item < nitems) rf_issue_rows<N>(gp, grow_of(item), G, bar);
    const float scale = 1.f / (float)N;
    const int kh = min(H / 2, kf - 1);
    for (uint32_t phase = 0; item < nitems; phase ^= 1) {
        if (!rf_wait_loads(bar, phase)) return;
        const long long next = item + gridDim.x;
        double rs = 0.0;
        const long long myrow = RSUM ? grow_of(item)(threadIdx.x / Lay::P) : -1ll;
        rf_forward_core<N, RSUM, PL::RZF>(G, X, tqs, [&] {
            if (next < nitems) {
                tc::fence_proxy_async();   // G was read (and zero rows written) through the generic proxy
                rf_issue_rows<N>(gp, grow_of(next), G, bar);
            }
        }, &rs);
        if (RSUM && myrow >= 0 && threadIdx.x % Lay::P == 0) rowsum[myrow] = rs;
        const long long field = item / nbpf;
        const int j0 = (int)(item - field * nbpf) * PR;
        const bool fin = field * nlat < lot;
        for (int it = threadIdx.x; it < PR * (kh + 1); it += blockDim.x) {
            const int pr = it % PR, k = it / PR, k2 = H - k, j = j0 + pr;
            if (!fin || j >= nlath) continue;
            cpx<float> *fr = reinterpret_cast<cpx<float> *>(fc) + field * nlat + j;   // E row; O is nlath further
            const cpx<float> *zn = X + pr * PL::RZF, *zs = X + (pr + PR) * PL::RZF;
            const cpx<float> an = zn[k], as = zs[k];
            if (k == 0) {
                const cpx<float> xn{(an.x + an.y) * scale, 0.f}, xs{(as.x + as.y) * scale, 0.f};
                fr[0] = cpx<float>{xn.x + xs.x, 0.f};
                fr[nlath] = cpx<float>{xn.x - xs.x, 0.f};
                continue;
            }
            const cpx<float> bn = zn[k2], bs = zs[k2], wk = rts[k];
            cpx<float> xn = rf_split(an, bn, wk, scale), xs = rf_split(as, bs, wk, scale);
            cpx<float> *fk = fr + (long long)k * f_ms;
            fk[0] = cpx<float>{xn.x + xs.x, xn.y + xs.y};
            fk[nlath] = cpx<float>{xn.x - xs.x, xn.y - xs.y};
            if (k2 < kf && k2 != k) {
                const cpx<float> wk2 = rts[k2];
                xn = rf_split(bn, an, wk2, scale);
                xs = rf_split(bs, as, wk2, scale);
                fk = fr + (long long)k2 * f_ms;
                fk[0] = cpx<float>{xn.x + xs.x, xn.y + xs.y};
                fk[nlath] = cpx<float>{xn.x - xs.x, xn.y - xs.y};
            }
        }
        __syncthreads();   // X is read before the next item's transposition writes it
        item = next;
    }
}

// rfft_inv_ct_body for the register-resident lengths: the block's
// coefficients c_k (k < kf) are staged k-major in shared memory by plain
// coalesced loads (a k's RB rows are one run of the m-major side); each thread
// forms the Z_k of its own q from c_k and c_{h-k}, takes their P-point DFTs,
// and after the transposition the Q-point DFT of its column; the grid rows
// leave through shared memory as one bulk store each
template <int N>
__device__ __forceinline__ void rfft_inv_rf_body(const float *fc, float *gp, long long lot, int kf, long long f_rs,
                                                 long long f_ms, const cpx<float> *__restrict__ w,
                                                 const cpx<float> *__restrict__ rt, long long blk) {
    using Lay = RfLayout<N>;
    constexpr int P = Lay::P, Q = Lay::Q, H = Lay::H, RB = Lay::RB, QP = Q / P;
    extern __shared__ __align__(16) unsigned char smraw[];
    const RfSmem<N> S(smraw);
    const long long row0 = blk * RB;
    const int rows = (int)min((long long)RB, lot - row0);
    const int t = threadIdx.x % P, r = threadIdx.x / P;
    pdl_trigger();
    rf_setup<N>(S, w, rt);
    pdl_wait();   // the coefficients come from the previous kernel
    const cpx<float> *fcc = reinterpret_cast<const cpx<float> *>(fc);
    cpx<float> *cs = S.r;   // c_k of row r at cs[k * RC + r]
    // the block's coefficients, k-major: plain loads, eight per thread in flight
    // (one k's rows are only RB x 8 bytes: bulk copies of that size were slower)
    {
        constexpr int U = 8;
        for (int i0 = threadIdx.x; i0 < kf * RB; i0 += U * (int)blockDim.x) {
            cpx<float> v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 + u * (int)blockDim.x, k = i / RB, rr = i - k * RB;
                v[u] = (i < kf * RB && rr < rows) ? fcc[(row0 + rr) * f_rs + (long long)k * f_ms] : cpx<float>{0.f, 0.f};
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 + u * (int)blockDim.x, k = i / RB, rr = i - k * RB;
                if (i < kf * RB) cs[k * Lay::RC + rr] = v[u];
            }
        }
        __syncthreads();
    }
    cpx<float> z[QP][P];
#pragma unroll
    for (int i = 0; i < QP; i++) {
        const int q = QP * t + i;
#pragma unroll
        for (int m = 0; m < P; m++) {
            const int k = q + Q * m, k2 = H - k;
            cpx<float> a{0.f, 0.f}, b{0.f, 0.f};
            if (k < kf) {
                a = cs[k * Lay::RC + r];
                if (k == 0) a.y = 0.f;
            }
            if (k > 0 && k2 < kf) b = cs[k2 * Lay::RC + r];
            // Z_k of the half-length complex sequence (c = 0 for k >= kf, the m = 0 imaginary part ignored)
            const cpx<float> E{a.x + b.x, a.y - b.y}, D{a.x - b.x, a.y + b.y};
            cpx<float> wk = S.rt[k];
            wk.y = -wk.y;
            const cpx<float> O = cmul(D, wk);
            z[i][m] = cpx<float>{E.x - O.y, E.y + O.x};
        }
        dft8<float, +1>(z[i]);
    }
    __syncthreads();   // the staged coefficients are read; the transposition overwrites them
    cpx<float> *x = S.r + r * Lay::RS;
#pragma unroll
    for (int i = 0; i < QP; i++)
#pragma unroll
        for (int u = 0; u < P; u++) x[u * Lay::RT + QP * t + i] = z[i][u];
    __syncthreads();
    cpx<float> v[Q];
    const cpx<float> *tq = S.tq + t * Lay::RT;
#pragma unroll
    for (int q = 0; q < Q; q += 2) {
        const float4 f = *reinterpret_cast<const float4 *>(x + t * Lay::RT + q);
        const float4 wq = *reinterpret_cast<const float4 *>(tq + q);
        v[q] = q ? cmul(cpx<float>{f.x, f.y}, cpx<float>{wq.x, -wq.y}) : cpx<float>{f.x, f.y};
        v[q + 1] = cmul(cpx<float>{f.z, f.w}, cpx<float>{wq.z, -wq.w});
    }
    dftQ<float, +1, Q>(v);
    __syncthreads();   // the transposition is read; the grid rows are staged over it
    cpx<float> *gs = S.r + r * Lay::RG + t;
#pragma unroll
    for (int j = 0; j < Q; j++) gs[P * j] = v[j];
    tc::fence_proxy_async();   // the staged rows feed the bulk stores
    __syncthreads();
    if (threadIdx.x < rows) {
        bulk_s2g(gp + (row0 + threadIdx.x) * N, S.r + threadIdx.x * Lay::RG, N * 4);
        bulk_commit_wait_read();
    }
}

// Persistent form of rfft_inv_rf_body.  A block sets up its twiddle tables
// once and walks the items blk = blockIdx.x, + gridDim.x, ... (RB rows each).
// The coefficients are staged k-major in their own region C by asynchronous
// 8-byte copies (cp.async), so the next item's copies are issued as soon as
// this item's coefficients are read and arrive while it is transformed and
// stored; the transposition and the staged grid rows use a second region.
__device__ __forceinline__ void cp_async8(void *dst_smem, const void *src_gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(tc::smem_u32(dst_smem)), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int N> struct RfIPLayout {
    using Lay = RfLayout<N>;
    static constexpr int RW = Lay::RS > Lay::RG ? Lay::RS : Lay::RG;
    // C takes kf x RC complex values (kf <= H); then the work region, the twiddle tables
    static __host__ __device__ size_t off_w(int kf) { return ((size_t)kf * Lay::RC * 8 + 15) & ~(size_t)15; }
    static __host__ __device__ size_t off_tq(int kf) { return off_w(kf) + (size_t)Lay::RB * RW * 8; }
    static __host__ __device__ size_t off_rt(int kf) { return off_tq(kf) + (size_t)Lay::P * Lay::RT * 8; }
    static __host__ __device__ size_t smem(int kf) { return off_rt(kf) + (size_t)Lay::H * 8; }
};

template <int N>
__global__ void __launch_bounds__(128) k_rfft_inv_rf_p(const float *fc, float *gp, long long lot, int kf,
                                                        long long f_rs, long long f_ms, long long nitems,
                                                        const cpx<float> *__restrict__ w,
                                                        const cpx<float> *__restrict__ rt) {
    using Lay = RfLayout<N>;
    using PL = RfIPLayout<N>;
    constexpr int P = Lay::P, Q = Lay::Q, H = Lay::H, RB = Lay::RB, QP = Q / P;
    extern __shared__ __align__(16) unsigned char smraw[];
    cpx<float> *cs = reinterpret_cast<cpx<float> *>(smraw);   // c_k of row r at cs[k * RC + r]
    cpx<float> *wk_s = reinterpret_cast<cpx<float> *>(smraw + PL::off_w(kf));
    cpx<float> *tqs = reinterpret_cast<cpx<float> *>(smraw + PL::off_tq(kf));
    cpx<float> *rts = reinterpret_cast<cpx<float> *>(smraw + PL::off_rt(kf));
    const int t = threadIdx.x % P, r = threadIdx.x / P;
    pdl_trigger();
    for (int i = threadIdx.x; i < P * Q; i += blockDim.x) {
        const int tt = i / Q, q = i - tt * Q;
        tqs[tt * Lay::RT + q] = w[tt * q];   // t q < h
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) rts[k] = rt[k];
    pdl_wait();   // the coefficients come from the previous kernel
    const cpx<float> *fcc = reinterpret_cast<const cpx<float> *>(fc);
    auto issue = [&](long long item) {
        const long long row0 = item * RB;
        const int rows = (int)min((long long)RB, lot - row0);
        for (int i = threadIdx.x; i < kf * RB; i += blockDim.x) {
            const int k = i / RB, rr = i - k * RB;
            cpx<float> *dst = cs + k * Lay::RC + rr;
            if (rr < rows) cp_async8(dst, fcc + (row0 + rr) * f_rs + (long long)k * f_ms);
            else *dst = cpx<float>{0.f, 0.f};
        }
        cp_async_commit();
    };
    long long item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        const long long row0 = item * RB;
        const int rows = (int)min((long long)RB, lot - row0);
        cp_async_wait_all();
        __syncthreads();   // this item's coefficients are in; the previous item's grid rows have left
        cpx<float> z[QP][P];
#pragma unroll
        for (int i = 0; i < QP; i++) {
            const int q = QP * t + i;
#pragma unroll
            for (int m = 0; m < P; m++) {
                const int k = q + Q * m, k2 = H - k;
                cpx<float> a{0.f, 0.f}, b{0.f, 0.f};
                if (k < kf) {
                    a = cs[k * Lay::RC + r];
                    if (k == 0) a.y = 0.f;
                }
                if (k > 0 && k2 < kf) b = cs[k2 * Lay::RC + r];
                // Z_k of the half-length complex sequence (c = 0 for k >= kf, the m = 0 imaginary part ignored)
                const cpx<float> E{a.x + b.x, a.y - b.y}, D{a.x - b.x, a.y + b.y};
                cpx<float> wk = rts[k];
                wk.y = -wk.y;
                const cpx<float> O = cmul(D, wk);
                z[i][m] = cpx<float>{E.x - O.y, E.y + O.x};
            }
            dft8<float, +1>(z[i]);
        }
        __syncthreads();   // the staged coefficients are read: the next item's copies may land
        if (item + gridDim.x < nitems) issue(item + gridDim.x);
        cpx<float> *x = wk_s + r * Lay::RS;
#pragma unroll
        for (int i = 0; i < QP; i++)
#pragma unroll
            for (int u = 0; u < P; u++) x[u * Lay::RT + QP * t + i] = z[i][u];
        __syncthreads();
        cpx<float> v[Q];
        const cpx<float> *tq = tqs + t * Lay::RT;
#pragma unroll
        for (int q = 0; q < Q; q += 2) {
            const float4 f = *reinterpret_cast<const float4 *>(x + t * Lay::RT + q);
            const float4 wq = *reinterpret_cast<const float4 *>(tq + q);
            v[q] = q ? cmul(cpx<float>{f.x, f.y}, cpx<float>{wq.x, -wq.y}) : cpx<float>{f.x, f.y};
            v[q + 1] = cmul(cpx<float>{f.z, f.w}, cpx<float>{wq.z, -wq.w});
        }
        dftQ<float, +1, Q>(v);
        __syncthreads();   // the transposition is read; the grid rows are staged over it
        cpx<float> *gs = wk_s + r * Lay::RG + t;
#pragma unroll
        for (int j = 0; j < Q; j++) gs[P * j] = v[j];
        tc::fence_proxy_async();   // the staged rows feed the bulk stores
        __syncthreads();
        if (threadIdx.x < rows) {
            bulk_s2g(gp + (row0 + threadIdx.x) * N, wk_s + threadIdx.x * Lay::RG, N * 4);
            bulk_commit_wait_read();
        }
    }
}

template <int N>
__global__ void __launch_bounds__(256) k_rfft_fwd_rf(const float *gp, float *fc, long long lot, int kf, long long f_rs,
                                                      long long f_ms, const cpx<float> *__restrict__ w,
                                                      const cpx<float> *__restrict__ rt) {
    rfft_fwd_rf_body<N>(gp, fc, lot, kf, f_rs, f_ms, w, rt, blockIdx.x);
}
template <int N>
__global__ void __launch_bounds__(256) k_rfft_inv_rf(const float *fc, float *gp, long long lot, int kf, long long f_rs,
                                                      long long f_ms, const cpx<float> *__restrict__ w,
                                                      const cpx<float> *__restrict__ rt) {
    rfft_inv_rf_body<N>(fc, gp, lot, kf, f_rs, f_ms, w, rt, blockIdx.x);
}
template <int N>
__global__ void __launch_bounds__(256) k_rfft_fwd_fold_rf(const float *gp, float *fc, int nlat, long long lot, int kf,
                                                           long long f_ms, const cpx<float> *__restrict__ w,
                                                           const cpx<float> *__restrict__ rt) {
    rfft_fwd_fold_rf_body<N>(gp, fc, nlat, lot, kf, f_ms, w, rt, blockIdx.x);
}

// ---------------------------------------------------------------- ensembles
// One launch transforms the rows of up to FFT_ENS_MAXSEG segments of different
// lengths (an uneven ensemble); block b belongs to the last segment whose
// first block is <= b.
struct FftEnsArgs {
    const float *in;
    float *out;
    long long lot, f_rs, f_ms;
    int n, kf, block0;
    int fold_nlat;          // forward only: > 0 writes the equator-folded layout (rfft_fwd_fold_body)
    const cpx<float> *w, *r;
};
struct FftEnsLaunch {
    FftEnsArgs seg[FFT_ENS_MAXSEG];
    int nseg;
};

template <bool FWD>
__global__ void __launch_bounds__(256) k_rfft_ens(const __grid_constant__ FftEnsLaunch P) {
    int s = 0;
    while (s + 1 < P.nseg && P.seg[s + 1].block0 <= (int)blockIdx.x) s++;
    const FftEnsArgs &S = P.seg[s];
    const long long blk = (long long)blockIdx.x - S.block0;
    switch (S.n) {
#define EXOTX_FFT_ENS_CASE(NN)                                                                                 \
    case NN:                                                                                                   \
        if (FWD && S.fold_nlat) rfft_fwd_fold_body<float, NN, ct_rows<float>(NN)>(S.in, S.out, S.fold_nlat, S.lot, S.kf, S.f_ms, S.w, S.r, blk); \
        else if (FWD) rfft_fwd_ct_body<float, NN, ct_rows<float>(NN)>(S.in, S.out, S.lot, S.kf, S.f_rs, S.f_ms, S.w, S.r, blk); \
        else rfft_inv_ct_body<float, NN, ct_rows<float>(NN)>(S.in, S.out, S.lot, S.kf, S.f_rs, S.f_ms, S.w, S.r, blk);    \
        break;
        EXOTX_FFT_ENS_CASE(64)
        EXOTX_FFT_ENS_CASE(128)
        EXOTX_FFT_ENS_CASE(192)
        EXOTX_FFT_ENS_CASE(256)
        EXOTX_FFT_ENS_CASE(320)
        EXOTX_FFT_ENS_CASE(512)
#undef EXOTX_FFT_ENS_CASE
        default: break;
    }
}
// the register-resident lengths (more registers per thread) in a launch of their own
template <bool FWD>
__global__ void __launch_bounds__(256) k_rfft_ens_rf(const __grid_constant__ FftEnsLaunch P) {
    int s = 0;
    while (s + 1 < P.nseg && P.seg[s + 1].block0 <= (int)blockIdx.x) s++;
    const FftEnsArgs &S = P.seg[s];
    const long long blk = (long long)blockIdx.x - S.block0;
    if (S.n == 384) {
        if (FWD && S.fold_nlat) rfft_fwd_fold_rf_body<384>(S.in, S.out, S.fold_nlat, S.lot, S.kf, S.f_ms, S.w, S.r, blk);
        else if (FWD) rfft_fwd_rf_body<384>(S.in, S.out, S.lot, S.kf, S.f_rs, S.f_ms, S.w, S.r, blk);
        else rfft_inv_rf_body<384>(S.in, S.out, S.lot, S.kf, S.f_rs, S.f_ms, S.w, S.r, blk);
    }
}

static bool ens_len(int n) {
    return n == 64 || n == 128 || n == 192 || n == 256 || n == 320 || n == 384 || n == 512;
}
static bool rf_len_host(int n) { return n == 384; }
static bool aligned16_(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// one launch over the segments whose lengths have (rf) or have not (!rf) a
// register-resident kernel
static exotx_status fft_ens_group(bool fwd, bool rf, const FftEnsSeg *segs, int nseg, cudaStream_t s) {
    FftEnsLaunch P;
    P.nseg = 0;
    int blocks = 0;
    size_t smem = 0;
    for (int i = 0; i < nseg; i++) {
        const FftEnsSeg &g = segs[i];
        if (rf_len_host(g.n) != rf) continue;
        exotx_status st;
        const FftTables *t = fft_tables(g.n, &st);
        if (!t) return st;
        const int rows = rf ? RfLayout<384>::RB : ct_rows<float>(g.n);
        FftEnsArgs &a = P.seg[P.nseg++];
        a.in = g.in; a.out = g.out; a.lot = g.lot; a.f_rs = g.f_rs; a.f_ms = g.f_ms; a.n = g.n; a.kf = g.kf;
        a.fold_nlat = fwd ? g.fold_nlat : 0;
        a.w = reinterpret_cast<const cpx<float> *>(t->w32);
        a.r = reinterpret_cast<const cpx<float> *>(t->r32);
        a.block0 = blocks;
        if (a.fold_nlat) {
            const int nbpf = (g.fold_nlat / 2 + rows / 2 - 1) / (rows / 2);
            blocks += (int)(g.lot / g.fold_nlat) * nbpf;
        } else {
            blocks += (int)((g.lot + rows - 1) / rows);
        }
        const int hp = g.n / 2 + 2 * (g.n / 32);   // padded row, as fpad_row
        smem = std::max(smem, rf ? RfLayout<384>::SMEM : 2 * (size_t)rows * hp * sizeof(cpx<float>));
    }
    if (blocks == 0) return EXOTX_OK;
    const int kid = fwd ? EXOTX_K_FFT_FORWARD : EXOTX_K_FFT_INVERSE;
    void (*k)(FftEnsLaunch) = rf ? (fwd ? k_rfft_ens_rf<true> : k_rfft_ens_rf<false>)
                                 : (fwd ? k_rfft_ens<true> : k_rfft_ens<false>);
    if (smem > 48 * 1024) EXOTX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaEvent_t ev = ktimer_start(kid, s);
    k<<<blocks, rf ? RfLayout<384>::NT : 256, smem, s>>>(P);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(kid, s, ev);
    return EXOTX_OK;
}

exotx_status fft_ens(bool fwd, const FftEnsSeg *segs, int nseg, cudaStream_t s) {
    if (nseg < 1 || nseg > FFT_ENS_MAXSEG) return EXOTX_BAD_ARG;
    for (int i = 0; i < nseg; i++) {
        const FftEnsSeg &g = segs[i];
        if (!ens_len(g.n)) return EXOTX_NOT_BUILT;
        if (!aligned16_(g.in) || !aligned16_(g.out)) return EXOTX_BAD_ARG;
        const int fold = fwd ? g.fold_nlat : 0;
        if (fold && (g.n != 2 * fold || g.lot % fold || g.f_rs != 1)) return EXOTX_BAD_ARG;
    }
    EXOTX_TRY(fft_ens_group(fwd, false, segs, nseg, s));
    return fft_ens_group(fwd, true, segs, nseg, s);
}

template <typename T, int N>
static exotx_status launch_ct(bool fwd, const T *in, T *out, long long lot, int kf, long long f_rs, long long f_ms,
                              const cpx<T> *w, const cpx<T> *r, cudaStream_t s) {
    constexpr int ROWS = ct_rows<T>(N);
    const size_t smem = 2 * ROWS * fpad_row<N / 2>() * sizeof(cpx<T>);
    const long long nb = (lot + ROWS - 1) / ROWS;
    const int kid = fwd ? EXOTX_K_FFT_FORWARD : EXOTX_K_FFT_INVERSE;
    if (fwd) {
        if (smem > 48 * 1024)
            EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_fwd_ct<T, N, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
    } else {
        if (smem > 48 * 1024)
            EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_inv_ct<T, N, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
    }
    cudaEvent_t ev = ktimer_start(kid, s);
    // dependent launch: the block set-up overlaps the previous kernel's tail
    if (fwd)
        EXOTX_CUDA(launch_pdl(k_rfft_fwd_ct<T, N, ROWS>, dim3((unsigned)nb), dim3(256), smem, s, in, out, lot, kf,
                              f_rs, f_ms, w, r));
    else
        EXOTX_CUDA(launch_pdl(k_rfft_inv_ct<T, N, ROWS>, dim3((unsigned)nb), dim3(256), smem, s, in, out, lot, kf,
                              f_rs, f_ms, w, r));
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(kid, s, ev);
    return EXOTX_OK;
}

// blocks of a kernel resident on the whole device at once (SMs x blocks per SM)
static exotx_status resident_slots(const void *kernel, int threads, size_t smem, int *slots) {
    int dev = 0, occ = 0, nsm = 0;
    EXOTX_CUDA(cudaGetDevice(&dev));
    EXOTX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem));
    EXOTX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    *slots = nsm * (occ < 1 ? 1 : occ);
    return EXOTX_OK;
}

template <int N>
static exotx_status launch_rf(bool fwd, const float *in, float *out, long long lot, int kf, long long f_rs,
                              long long f_ms, const cpx<float> *w, const cpx<float> *r, cudaStream_t s) {
    using Lay = RfLayout<N>;
    const long long nb = (lot + Lay::RB - 1) / Lay::RB;
    const int kid = fwd ? EXOTX_K_FFT_FORWARD : EXOTX_K_FFT_INVERSE;
    if (fwd)
        EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_fwd_rf<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::SMEM));
    else if (kf > Lay::H)
        EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_inv_rf<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::SMEM));
    long long grid = nb;
    size_t smem_p = 0;
    if (!fwd && kf <= Lay::H) {   // persistent form: one block per resident slot
        smem_p = RfIPLayout<N>::smem(kf);
        EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_inv_rf_p<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_p));
        int slots = 0;
        EXOTX_TRY(resident_slots((const void *)k_rfft_inv_rf_p<N>, Lay::NT, smem_p, &slots));
        grid = std::min<long long>(nb, slots);
    }
    cudaEvent_t ev = ktimer_start(kid, s);
    if (fwd)
        EXOTX_CUDA(launch_pdl(k_rfft_fwd_rf<N>, dim3((unsigned)nb), dim3(Lay::NT), Lay::SMEM, s, in, out, lot, kf, f_rs,
                              f_ms, w, r));
    else if (smem_p)
        EXOTX_CUDA(launch_pdl(k_rfft_inv_rf_p<N>, dim3((unsigned)grid), dim3(Lay::NT), smem_p, s, in, out, lot, kf,
                              f_rs, f_ms, nb, w, r));
    else
        EXOTX_CUDA(launch_pdl(k_rfft_inv_rf<N>, dim3((unsigned)nb), dim3(Lay::NT), Lay::SMEM, s, in, out, lot, kf, f_rs,
                              f_ms, w, r));
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(kid, s, ev);
    return EXOTX_OK;
}

// returns EXOTX_NOT_BUILT when n has no specialised kernel
template <typename T>
static exotx_status dispatch_ct(bool fwd, int n, const T *in, T *out, long long lot, int kf, long long f_rs,
                                long long f_ms, const cpx<T> *w, const cpx<T> *r, cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {   // single precision: register-resident kernels where built
        if (n == 384) return launch_rf<384>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
    }
    switch (n) {
        case 64: return launch_ct<T, 64>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 128: return launch_ct<T, 128>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 192: return launch_ct<T, 192>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 256: return launch_ct<T, 256>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 320: return launch_ct<T, 320>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 384: return launch_ct<T, 384>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
        case 512: return launch_ct<T, 512>(fwd, in, out, lot, kf, f_rs, f_ms, w, r, s);
    }
    return EXOTX_NOT_BUILT;
}

// ----------------------------------------------------------------- tables
static bool factor_h(int h, int *fac, int *nfac) {
    int k = 0, r = h;
    while (r % 8 == 0 && r > 8) { fac[k++] = 8; r /= 8; }
    while (r % 4 == 0) { fac[k++] = 4; r /= 4; }
    while (r % 2 == 0) { fac[k++] = 2; r /= 2; }
    while (r % 3 == 0) { fac[k++] = 3; r /= 3; }
    while (r % 5 == 0) { fac[k++] = 5; r /= 5; }
    if (r == 8) { fac[k++] = 8; r = 1; }
    if (r != 1 || k > 16) return false;
    *nfac = k;
    return true;
}

static std::mutex g_fft_mu;
static std::map<int, FftTables *> g_fft_cache;

const FftTables *fft_tables(int n, exotx_status *st) {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    auto it = g_fft_cache.find(n);
    if (it != g_fft_cache.end()) { *st = EXOTX_OK; return it->second; }
    if (!exotx_fft_supported(n)) { *st = EXOTX_UNSUPPORTED_N; return nullptr; }
    FftTables *t = new FftTables();
    t->n = n;
    t->h = n / 2;
    factor_h(t->h, t->fac, &t->nfac);
    int h = t->h;
    // twiddles from exact integer angles, evaluated in long double
    std::vector<double> w64(2 * h), r64(2 * (h + 1));
    std::vector<float> w32(2 * h), r32(2 * (h + 1));
    const long double PI_L = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < h; k++) {
        long double a = -2.0L * PI_L * (long double)k / (long double)h;
        w64[2 * k] = (double)cosl(a); w64[2 * k + 1] = (double)sinl(a);
        w32[2 * k] = (float)cosl(a); w32[2 * k + 1] = (float)sinl(a);
    }
    for (int k = 0; k <= h; k++) {
        long double a = -2.0L * PI_L * (long double)k / (long double)n;
        r64[2 * k] = (double)cosl(a); r64[2 * k + 1] = (double)sinl(a);
        r32[2 * k] = (float)cosl(a); r32[2 * k + 1] = (float)sinl(a);
    }
    bool ok = cudaMalloc(&t->w64, sizeof(double) * 2 * h) == cudaSuccess &&
              cudaMalloc(&t->w32, sizeof(float) * 2 * h) == cudaSuccess &&
              cudaMalloc(&t->r64, sizeof(double) * 2 * (h + 1)) == cudaSuccess &&
              cudaMalloc(&t->r32, sizeof(float) * 2 * (h + 1)) == cudaSuccess;
    ok = ok && cudaMemcpy(t->w64, w64.data(), sizeof(double) * 2 * h, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(t->w32, w32.data(), sizeof(float) * 2 * h, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(t->r64, r64.data(), sizeof(double) * 2 * (h + 1), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(t->r32, r32.data(), sizeof(float) * 2 * (h + 1), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        cudaFree(t->w64); cudaFree(t->w32); cudaFree(t->r64); cudaFree(t->r32);
        delete t;
        *st = EXOTX_NO_MEM;
        return nullptr;
    }
    g_fft_cache[n] = t;
    *st = EXOTX_OK;
    return t;
}

template <typename T> static const cpx<T> *wt(const FftTables *t);
template <> const cpx<double> *wt<double>(const FftTables *t) { return reinterpret_cast<const cpx<double> *>(t->w64); }
template <> const cpx<float> *wt<float>(const FftTables *t) { return reinterpret_cast<const cpx<float> *>(t->w32); }
template <typename T> static const cpx<T> *rt(const FftTables *t);
template <> const cpx<double> *rt<double>(const FftTables *t) { return reinterpret_cast<const cpx<double> *>(t->r64); }
template <> const cpx<float> *rt<float>(const FftTables *t) { return reinterpret_cast<const cpx<float> *>(t->r32); }

template <typename T>
static FftLaunch make_launch(const FftTables *t, long long lot, int kf, long long f_rs, long long f_ms,
                             size_t *smem) {
    FftLaunch L;
    L.n = t->n; L.h = t->h; L.nfac = t->nfac;
    for (int i = 0; i < 16; i++) L.fac[i] = t->fac[i];
    L.lot = lot; L.kf = kf; L.f_rs = f_rs; L.f_ms = f_ms;
    size_t per_row = 2 * (size_t)t->n * sizeof(T);
    int r = (int)((40 * 1024) / per_row);
    r = r < 1 ? 1 : (r > 16 ? 16 : r);
    L.rows_per_block = r;
    *smem = per_row * r;
    return L;
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T>
static exotx_status set_smem(const void *fn, size_t smem) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_status(e);
    }
    return EXOTX_OK;
}

// Fourier layout helper: row-major reference layout (row stride n/2, m stride 1)
template <typename T>
exotx_status fft_forward_l(const T *in, T *out, int n, long long lot, int kout, long long f_rs, long long f_ms,
                           cudaStream_t s) {
    exotx_status st;
    const FftTables *t = fft_tables(n, &st);
    if (!t) return st;
    if (lot <= 0) return EXOTX_OK;
    if (aligned16(in) && aligned16(out)) {
        exotx_status sc = dispatch_ct<T>(true, n, in, out, lot, kout, f_rs, f_ms, wt<T>(t), rt<T>(t), s);
        if (sc != EXOTX_NOT_BUILT) return sc;
    }
    size_t smem;
    FftLaunch L = make_launch<T>(t, lot, kout, f_rs, f_ms, &smem);
    EXOTX_TRY(set_smem<T>((const void *)k_rfft_forward<T>, smem));
    long long nb = (lot + L.rows_per_block - 1) / L.rows_per_block;
    cudaEvent_t ev = ktimer_start(EXOTX_K_FFT_FORWARD, s);
    k_rfft_forward<T><<<(unsigned)nb, 256, smem, s>>>(in, out, L, wt<T>(t), rt<T>(t));
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_FFT_FORWARD, s, ev);
    return EXOTX_OK;
}

template <typename T>
exotx_status fft_inverse_l(const T *in, T *out, int n, long long lot, int kin, long long f_rs, long long f_ms,
                           cudaStream_t s) {
    exotx_status st;
    const FftTables *t = fft_tables(n, &st);
    if (!t) return st;
    if (lot <= 0) return EXOTX_OK;
    if (aligned16(in) && aligned16(out)) {
        exotx_status sc = dispatch_ct<T>(false, n, in, out, lot, kin, f_rs, f_ms, wt<T>(t), rt<T>(t), s);
        if (sc != EXOTX_NOT_BUILT) return sc;
    }
    size_t smem;
    FftLaunch L = make_launch<T>(t, lot, kin, f_rs, f_ms, &smem);
    EXOTX_TRY(set_smem<T>((const void *)k_rfft_inverse<T>, smem));
    long long nb = (lot + L.rows_per_block - 1) / L.rows_per_block;
    cudaEvent_t ev = ktimer_start(EXOTX_K_FFT_INVERSE, s);
    k_rfft_inverse<T><<<(unsigned)nb, 256, smem, s>>>(in, out, L, wt<T>(t), rt<T>(t));
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_FFT_INVERSE, s, ev);
    return EXOTX_OK;
}

template exotx_status fft_forward_l<double>(const double *, double *, int, long long, int, long long, long long,
                                            cudaStream_t);
template exotx_status fft_forward_l<float>(const float *, float *, int, long long, int, long long, long long,
                                           cudaStream_t);

template <int N>
static exotx_status launch_fold(const float *in, float *out, int nlat, long long lot, int kf, long long f_ms,
                                const cpx<float> *w, const cpx<float> *r, double *rowsum, cudaStream_t s) {
    if (rowsum && !rf_len<N>()) return EXOTX_NOT_BUILT;
    if constexpr (rf_len<N>()) {
        using Lay = RfLayout<N>;
        using PL = RfPLayout<N>;
        const int nbpf = (nlat / 2 + Lay::RB / 2 - 1) / (Lay::RB / 2);
        const long long nb = (lot / nlat) * nbpf;
        auto kern = rowsum ? k_rfft_fwd_fold_rf_p<N, true> : k_rfft_fwd_fold_rf_p<N, false>;
        EXOTX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
        int slots = 0;
        EXOTX_TRY(resident_slots((const void *)kern, Lay::NT, PL::SMEM, &slots));
        const long long grid = std::min<long long>(nb, slots);
        cudaEvent_t ev = ktimer_start(EXOTX_K_FFT_FORWARD, s);
        EXOTX_CUDA(launch_pdl(kern, dim3((unsigned)grid), dim3(Lay::NT), PL::SMEM, s, in, out, nlat, lot, kf, f_ms, nb,
                              w, r, rowsum));
        EXOTX_CHECK_LAUNCH();
        ktimer_stop(EXOTX_K_FFT_FORWARD, s, ev);
        return EXOTX_OK;
    }
    constexpr int ROWS = ct_rows<float>(N);
    const size_t smem = 2 * ROWS * fpad_row<N / 2>() * sizeof(cpx<float>);
    const int nbpf = (nlat / 2 + ROWS / 2 - 1) / (ROWS / 2);
    const long long nb = (lot / nlat) * nbpf;
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_fwd_fold<float, N, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    cudaEvent_t ev = ktimer_start(EXOTX_K_FFT_FORWARD, s);
    EXOTX_CUDA(launch_pdl(k_rfft_fwd_fold<float, N, ROWS>, dim3((unsigned)nb), dim3(256), smem, s, in, out, nlat, lot,
                          kf, f_ms, w, r));
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_FFT_FORWARD, s, ev);
    return EXOTX_OK;
}

// forward transform of lot = fields x nlat grid rows of length n = 2 nlat into
// the equator-folded m-major layout (rfft_fwd_fold_body); EXOTX_NOT_BUILT when
// n has no specialised kernel or the buffers are not 16-byte aligned
bool fft_fold_rowsum(int n) { return n == 384; }   // the register-resident lengths (RfShape)

exotx_status fft_forward_fold(const float *in, float *out, int n, int nlat, long long lot, int kf, long long f_ms,
                              double *rowsum, cudaStream_t s) {
    if (n != 2 * nlat || nlat < 2 || lot % nlat) return EXOTX_BAD_ARG;
    exotx_status st;
    const FftTables *t = fft_tables(n, &st);
    if (!t) return st;
    if (lot <= 0) return EXOTX_OK;
    if (!aligned16(in) || !aligned16(out)) return EXOTX_NOT_BUILT;
    const cpx<float> *w = wt<float>(t), *r = rt<float>(t);
    switch (n) {
        case 64: return launch_fold<64>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 128: return launch_fold<128>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 192: return launch_fold<192>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 256: return launch_fold<256>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 320: return launch_fold<320>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 384: return launch_fold<384>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
        case 512: return launch_fold<512>(in, out, nlat, lot, kf, f_ms, w, r, rowsum, s);
    }
    return EXOTX_NOT_BUILT;
}
template exotx_status fft_inverse_l<double>(const double *, double *, int, long long, int, long long, long long,
                                            cudaStream_t);
template exotx_status fft_inverse_l<float>(const float *, float *, int, long long, int, long long, long long,
                                           cudaStream_t);

exotx_status fft_error_reset(cudaStream_t s) {
    int zero = 0;
    EXOTX_CUDA(cudaMemcpyToSymbolAsync(g_fft_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
    return EXOTX_OK;
}
exotx_status fft_error_read(int *err, cudaStream_t s) {
    EXOTX_CUDA(cudaMemcpyFromSymbolAsync(err, g_fft_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    EXOTX_CUDA(cudaStreamSynchronize(s));
    return EXOTX_OK;
}

// ----------------------------------------------- caller-supplied twiddle tables
// The twiddle values the cached tables hold (same long-double evaluation, so
// the transforms agree bit for bit), written into caller buffers of h and h+1
// complex values.
template <typename T>
void fft_twiddles_host(int n, T *w, T *r) {
    const int h = n / 2;
    const long double PI_L = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < h; k++) {
        long double a = -2.0L * PI_L * (long double)k / (long double)h;
        w[2 * k] = (T)cosl(a); w[2 * k + 1] = (T)sinl(a);
    }
    for (int k = 0; k <= h; k++) {
        long double a = -2.0L * PI_L * (long double)k / (long double)n;
        r[2 * k] = (T)cosl(a); r[2 * k + 1] = (T)sinl(a);
    }
}
template void fft_twiddles_host<double>(int, double *, double *);
template void fft_twiddles_host<float>(int, float *, float *);

// fft_forward_l with the twiddles in caller memory (device pointers laid out
// as fft_twiddles_host writes them); launches the same kernels and allocates
// nothing.
template <typename T>
exotx_status fft_forward_tw(const T *in, T *out, int n, long long lot, int kout, long long f_rs, long long f_ms,
                            const T *w, const T *r, cudaStream_t s) {
    if (!exotx_fft_supported(n)) return EXOTX_UNSUPPORTED_N;
    if (lot <= 0) return EXOTX_OK;
    const cpx<T> *wc = reinterpret_cast<const cpx<T> *>(w), *rc = reinterpret_cast<const cpx<T> *>(r);
    if (aligned16(in) && aligned16(out)) {
        exotx_status sc = dispatch_ct<T>(true, n, in, out, lot, kout, f_rs, f_ms, wc, rc, s);
        if (sc != EXOTX_NOT_BUILT) return sc;
    }
    FftTables t;  // radix schedule only
    t.n = n;
    t.h = n / 2;
    factor_h(t.h, t.fac, &t.nfac);
    size_t smem;
    FftLaunch L = make_launch<T>(&t, lot, kout, f_rs, f_ms, &smem);
    EXOTX_TRY(set_smem<T>((const void *)k_rfft_forward<T>, smem));
    long long nb = (lot + L.rows_per_block - 1) / L.rows_per_block;
    cudaEvent_t ev = ktimer_start(EXOTX_K_FFT_FORWARD, s);
    k_rfft_forward<T><<<(unsigned)nb, 256, smem, s>>>(in, out, L, wc, rc);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_FFT_FORWARD, s, ev);
    return EXOTX_OK;
}
template exotx_status fft_forward_tw<double>(const double *, double *, int, long long, int, long long, long long,
                                             const double *, const double *, cudaStream_t);
template exotx_status fft_forward_tw<float>(const float *, float *, int, long long, int, long long, long long,
                                            const float *, const float *, cudaStream_t);

}  // namespace exotx

EXOTX_API int exotx_fft_supported(int n) {
    if (n < 4 || n > 4096 || (n & 1)) return 0;
    int h = n / 2, fac[16], nfac;
    return exotx::factor_h(h, fac, &nfac) ? 1 : 0;
}
