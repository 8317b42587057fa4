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
        EXOTX_FFT_ENS_CASE(384)
        EXOTX_FFT_ENS_CASE(512)
#undef EXOTX_FFT_ENS_CASE
        default: break;
    }
}

static bool ens_len(int n) {
    return n == 64 || n == 128 || n == 192 || n == 256 || n == 320 || n == 384 || n == 512;
}
static bool aligned16_(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

exotx_status fft_ens(bool fwd, const FftEnsSeg *segs, int nseg, cudaStream_t s) {
    if (nseg < 1 || nseg > FFT_ENS_MAXSEG) return EXOTX_BAD_ARG;
    FftEnsLaunch P;
    P.nseg = nseg;
    int blocks = 0;
    size_t smem = 0;
    for (int i = 0; i < nseg; i++) {
        const FftEnsSeg &g = segs[i];
        if (!ens_len(g.n)) return EXOTX_NOT_BUILT;
        if (!aligned16_(g.in) || !aligned16_(g.out)) return EXOTX_BAD_ARG;
        exotx_status st;
        const FftTables *t = fft_tables(g.n, &st);
        if (!t) return st;
        const int rows = ct_rows<float>(g.n);
        FftEnsArgs &a = P.seg[i];
        a.in = g.in; a.out = g.out; a.lot = g.lot; a.f_rs = g.f_rs; a.f_ms = g.f_ms; a.n = g.n; a.kf = g.kf;
        a.fold_nlat = fwd ? g.fold_nlat : 0;
        if (a.fold_nlat && (g.n != 2 * g.fold_nlat || g.lot % g.fold_nlat || g.f_rs != 1)) return EXOTX_BAD_ARG;
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
        smem = std::max(smem, 2 * (size_t)rows * hp * sizeof(cpx<float>));
    }
    if (blocks == 0) return EXOTX_OK;
    const int kid = fwd ? EXOTX_K_FFT_FORWARD : EXOTX_K_FFT_INVERSE;
    if (fwd) {
        if (smem > 48 * 1024)
            EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_ens<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    } else if (smem > 48 * 1024) {
        EXOTX_CUDA(cudaFuncSetAttribute(k_rfft_ens<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    cudaEvent_t ev = ktimer_start(kid, s);
    if (fwd) k_rfft_ens<true><<<blocks, 256, smem, s>>>(P);
    else k_rfft_ens<false><<<blocks, 256, smem, s>>>(P);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(kid, s, ev);
    return EXOTX_OK;
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

// returns EXOTX_NOT_BUILT when n has no specialised kernel
template <typename T>
static exotx_status dispatch_ct(bool fwd, int n, const T *in, T *out, long long lot, int kf, long long f_rs,
                                long long f_ms, const cpx<T> *w, const cpx<T> *r, cudaStream_t s) {
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
                                const cpx<float> *w, const cpx<float> *r, cudaStream_t s) {
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
exotx_status fft_forward_fold(const float *in, float *out, int n, int nlat, long long lot, int kf, long long f_ms,
                              cudaStream_t s) {
    if (n != 2 * nlat || nlat < 2 || lot % nlat) return EXOTX_BAD_ARG;
    exotx_status st;
    const FftTables *t = fft_tables(n, &st);
    if (!t) return st;
    if (lot <= 0) return EXOTX_OK;
    if (!aligned16(in) || !aligned16(out)) return EXOTX_NOT_BUILT;
    const cpx<float> *w = wt<float>(t), *r = rt<float>(t);
    switch (n) {
        case 64: return launch_fold<64>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 128: return launch_fold<128>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 192: return launch_fold<192>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 256: return launch_fold<256>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 320: return launch_fold<320>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 384: return launch_fold<384>(in, out, nlat, lot, kf, f_ms, w, r, s);
        case 512: return launch_fold<512>(in, out, nlat, lot, kf, f_ms, w, r, s);
    }
    return EXOTX_NOT_BUILT;
}
template exotx_status fft_inverse_l<double>(const double *, double *, int, long long, int, long long, long long,
                                            cudaStream_t);
template exotx_status fft_inverse_l<float>(const float *, float *, int, long long, int, long long, long long,
                                           cudaStream_t);

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
