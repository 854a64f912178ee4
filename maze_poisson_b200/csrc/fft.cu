// Spectral Poisson solve phi = IFFT( FFT(q) * ig2 ) on an n^3 periodic grid, written as
// five passes over an n x n x (n/2+1) complex spectrum in HBM:
//   K  : r2c along k (rows of n reals -> n/2+1 complex)
//   J  : forward along j
//   I  : forward along i, multiply by ig2, inverse along i (one read, one write)
//   J' : inverse along j
//   K' : c2r along k
// For n = 64, 128 and 256 each 1-D transform runs in registers (see solve_reg); other
// sizes run each 1-D transform in shared memory as a mixed-radix (4, 2, 3) Stockham FFT.
// Both use an accurate twiddle table (sincospi). Reference semantics (library/src/grid_fft.c:65-125,
// fftw_wrap.c:166-189): ig2 = 4 pi / (h^3 n^3) / (k^2 + 1e-10) with continuous
// k = 2 pi m / L, the unnormalised inverse transform, and the DC term left unmultiplied.
#include "fft.cuh"

namespace mzb {
namespace {

constexpr int kFftThreads = 256;
constexpr int kRowsPerBlock = 4;   // pass K: rows per block
constexpr int kColsPerBlock = 8;   // passes J/I: spectrum columns per block
constexpr int kMaxStages = 16;

struct Radices {
    int nst;
    int r[kMaxStages];
};

Radices plan_radices(int n) {
    Radices p{};
    int m = n;
    while (m % 4 == 0) { p.r[p.nst++] = 4; m /= 4; }
    while (m % 2 == 0) { p.r[p.nst++] = 2; m /= 2; }
    while (m % 3 == 0) { p.r[p.nst++] = 3; m /= 3; }
    if (m != 1) fatal("FFT: grid size must be of the form 2^a 3^b");
    return p;
}

// Batched Stockham FFT in shared memory. Element e of sequence b lives at b*bs + e*es in
// (re, im); (re2, im2) is scratch of the same size. Returns true if the result ended in
// the scratch buffers. INV selects the +i (inverse, unnormalised) transform.
template <bool INV>
__device__ bool fft_batch(double* re, double* im, double* re2, double* im2, int n, int nb, int es,
                          int bs, const double* wre, const double* wim, const Radices& rd) {
    double *ir = re, *ii = im, *orr = re2, *oi = im2;
    int Ns = 1;
    for (int st = 0; st < rd.nst; st++) {
        const int R = rd.r[st];
        const int nr = n / R;
        const int tw_step = n / (Ns * R);
        for (int idx = threadIdx.x; idx < nb * nr; idx += blockDim.x) {
            const int b = idx / nr, j = idx - b * nr;
            const int jm = j % Ns;
            double xr[4], xi[4];
            for (int r = 0; r < R; r++) {
                const int a = b * bs + (j + r * nr) * es;
                double vr = ir[a], vi = ii[a];
                const int t = (jm * r * tw_step) % n;
                if (t != 0) {
                    const double cr = wre[t], ci = INV ? -wim[t] : wim[t];
                    const double nr2 = fma(vr, cr, -vi * ci), ni2 = fma(vr, ci, vi * cr);
                    vr = nr2;
                    vi = ni2;
                }
                xr[r] = vr;
                xi[r] = vi;
            }
            double yr[4], yi[4];
            if (R == 2) {
                yr[0] = xr[0] + xr[1]; yi[0] = xi[0] + xi[1];
                yr[1] = xr[0] - xr[1]; yi[1] = xi[0] - xi[1];
            } else if (R == 4) {
                const double ar = xr[0] + xr[2], ai = xi[0] + xi[2];
                const double br = xr[0] - xr[2], bi = xi[0] - xi[2];
                const double cr = xr[1] + xr[3], ci = xi[1] + xi[3];
                // d = -i (x1 - x3) forward, +i (x1 - x3) inverse
                const double er = xr[1] - xr[3], ei = xi[1] - xi[3];
                const double dr = INV ? -ei : ei, di = INV ? er : -er;
                yr[0] = ar + cr; yi[0] = ai + ci;
                yr[1] = br + dr; yi[1] = bi + di;
                yr[2] = ar - cr; yi[2] = ai - ci;
                yr[3] = br - dr; yi[3] = bi - di;
            } else {  // R == 3
                const double s3 = 0.86602540378443864676;  // sqrt(3)/2
                const double tr = xr[1] + xr[2], ti = xi[1] + xi[2];
                const double ur = fma(-0.5, tr, xr[0]), ui = fma(-0.5, ti, xi[0]);
                const double dr = xr[1] - xr[2], di = xi[1] - xi[2];
                // v = -i s3 (x1 - x2) forward, +i s3 (x1 - x2) inverse
                const double vr = INV ? -s3 * di : s3 * di, vi = INV ? s3 * dr : -s3 * dr;
                yr[0] = xr[0] + tr; yi[0] = xi[0] + ti;
                yr[1] = ur + vr; yi[1] = ui + vi;
                yr[2] = ur - vr; yi[2] = ui - vi;
            }
            const int dst = (j / Ns) * Ns * R + jm;
            for (int r = 0; r < R; r++) {
                const int a = b * bs + (dst + r * Ns) * es;
                orr[a] = yr[r];
                oi[a] = yi[r];
            }
        }
        __syncthreads();
        double* t0 = ir; ir = orr; orr = t0;
        double* t1 = ii; ii = oi; oi = t1;
        Ns *= R;
    }
    return (rd.nst & 1) != 0;
}

__device__ __forceinline__ void load_twiddles(double* wre, double* wim, const double2* W, int n) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        wre[t] = W[t].x;
        wim[t] = W[t].y;
    }
}

__global__ void k_twiddles(double2* W, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double s, c;
    sincospi(2.0 * t / n, &s, &c);
    W[t] = make_double2(c, -s);  // exp(-2 pi i t / n)
}

// Continuous wavenumbers exactly as grid_fft.c:94-102: freq[m] = (2 pi m)/L for
// m <= n/2 (n/2+1 values), (2 pi (m - n))/L from m = n/2 (even n) or (n+1)/2 (odd n).
__global__ void k_freqs(double* freq, double* rfreq, int n, double L) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = n / 2 + 1;
    const double pi2 = 2 * kPi;
    if (m < nh) rfreq[m] = pi2 * m / L;
    if (m < n) {
        const int first_neg = (n % 2) ? nh : nh - 1;
        freq[m] = m >= first_neg ? pi2 * (m - n) / L : pi2 * m / L;
    }
}

// ---- pass K: r2c along k ----
__global__ void __launch_bounds__(kFftThreads) k_pass_k_fwd(const double* __restrict__ in,
                                                             double2* __restrict__ spec,
                                                             const double2* __restrict__ W, int n,
                                                             Radices rd) {
    extern __shared__ double sm[];
    const int nh = n / 2 + 1, RB = kRowsPerBlock;
    double *wre = sm, *wim = wre + n, *re = wim + n, *im = re + RB * n, *re2 = im + RB * n,
           *im2 = re2 + RB * n;
    load_twiddles(wre, wim, W, n);
    const long rows = (long)n * n, row0 = (long)blockIdx.x * RB;
    for (int e = threadIdx.x; e < RB * n; e += blockDim.x) {
        const int b = e / n, k = e - b * n;
        const long row = row0 + b;
        re[e] = row < rows ? in[row * n + k] : 0.0;
        im[e] = 0.0;
    }
    __syncthreads();
    const bool sw = fft_batch<false>(re, im, re2, im2, n, RB, 1, n, wre, wim, rd);
    const double *orr = sw ? re2 : re, *oi = sw ? im2 : im;
    for (int e = threadIdx.x; e < RB * nh; e += blockDim.x) {
        const int b = e / nh, k = e - b * nh;
        const long row = row0 + b;
        if (row < rows) spec[row * nh + k] = make_double2(orr[b * n + k], oi[b * n + k]);
    }
}

// ---- pass K': c2r along k ----
__global__ void __launch_bounds__(kFftThreads) k_pass_k_inv(const double2* __restrict__ spec,
                                                             double* __restrict__ out,
                                                             const double2* __restrict__ W, int n,
                                                             Radices rd) {
    extern __shared__ double sm[];
    const int nh = n / 2 + 1, RB = kRowsPerBlock;
    double *wre = sm, *wim = wre + n, *re = wim + n, *im = re + RB * n, *re2 = im + RB * n,
           *im2 = re2 + RB * n;
    load_twiddles(wre, wim, W, n);
    const long rows = (long)n * n, row0 = (long)blockIdx.x * RB;
    for (int e = threadIdx.x; e < RB * n; e += blockDim.x) {
        const int b = e / n, k = e - b * n;
        const long row = row0 + b;
        double2 v = make_double2(0.0, 0.0);
        if (row < rows) {
            if (k < nh) v = spec[row * nh + k];
            else {
                v = spec[row * nh + (n - k)];
                v.y = -v.y;
            }
        }
        re[e] = v.x;
        im[e] = v.y;
    }
    __syncthreads();
    const bool sw = fft_batch<true>(re, im, re2, im2, n, RB, 1, n, wre, wim, rd);
    const double* orr = sw ? re2 : re;
    for (int e = threadIdx.x; e < RB * n; e += blockDim.x) {
        const int b = e / n, k = e - b * n;
        const long row = row0 + b;
        if (row < rows) out[row * n + k] = orr[e];
    }
}

// ---- passes J / I: columns of the spectrum along axis j (fixed i) or i (fixed j) ----
// MODE 0: forward along j; 1: inverse along j; 2: forward along i, multiply, inverse along i
template <int MODE>
__global__ void __launch_bounds__(kFftThreads) k_pass_cols(double2* __restrict__ spec,
                                                            const double2* __restrict__ W, int n,
                                                            Radices rd, const double* __restrict__ freq,
                                                            const double* __restrict__ rfreq,
                                                            double cst) {
    extern __shared__ double sm[];
    const int nh = n / 2 + 1, TK = kColsPerBlock;
    double *wre = sm, *wim = wre + n, *re = wim + n, *im = re + TK * n, *re2 = im + TK * n,
           *im2 = re2 + TK * n;
    load_twiddles(wre, wim, W, n);
    const int ntk = (nh + TK - 1) / TK;
    const int fixed = blockIdx.x / ntk, kh0 = (blockIdx.x % ntk) * TK;
    const long n2h = (long)n * nh;
    // element e (0..n) of column kk: (i = fixed, j = e) for MODE 0/1, (i = e, j = fixed) MODE 2
    auto gaddr = [&](int e, int kk) -> long {
        return MODE == 2 ? (long)e * n2h + (long)fixed * nh + kh0 + kk
                         : (long)fixed * n2h + (long)e * nh + kh0 + kk;
    };
    for (int x = threadIdx.x; x < TK * n; x += blockDim.x) {
        const int e = x / TK, kk = x - e * TK;
        double2 v = make_double2(0.0, 0.0);
        if (kh0 + kk < nh) v = spec[gaddr(e, kk)];
        re[x] = v.x;
        im[x] = v.y;
    }
    __syncthreads();
    bool sw;
    if (MODE == 1) sw = fft_batch<true>(re, im, re2, im2, n, TK, TK, 1, wre, wim, rd);
    else sw = fft_batch<false>(re, im, re2, im2, n, TK, TK, 1, wre, wim, rd);
    double *orr = sw ? re2 : re, *oi = sw ? im2 : im;
    if (MODE == 2) {
        // ig2(i, j, kh) = cst / ((freq_i^2 + freq_j^2) + rfreq_kh^2 + 1e-10), DC untouched
        const double fj = freq[fixed];
        for (int x = threadIdx.x; x < TK * n; x += blockDim.x) {
            const int e = x / TK, kk = x - e * TK, kh = kh0 + kk;
            if (kh >= nh) continue;
            if (e == 0 && fixed == 0 && kh == 0) continue;
            const double fi = freq[e], rk = rfreq[kh];
            const double f1 = fi * fi;
            const double f2 = f1 + fj * fj;
            const double g = cst / (f2 + rk * rk + 1E-10);
            orr[x] *= g;
            oi[x] *= g;
        }
        __syncthreads();
        double *sr = sw ? re : re2, *si = sw ? im : im2;
        sw = fft_batch<true>(orr, oi, sr, si, n, TK, TK, 1, wre, wim, rd);
        if (sw) { orr = sr; oi = si; }
    }
    for (int x = threadIdx.x; x < TK * n; x += blockDim.x) {
        const int e = x / TK, kk = x - e * TK;
        if (kh0 + kk < nh) spec[gaddr(e, kk)] = make_double2(orr[x], oi[x]);
    }
}

// ---- register-resident transforms for n = 64, 128, 256 ----
//
// A length-N transform is split N = N1 x N2 (Cooley-Tukey, four-step): N2 threads work it,
// thread t holding x[n1 N2 + t] for n1 < N1; each forms a length-N1 DFT in registers,
// multiplies by W_N^(t k1), the partial results are exchanged through shared memory, and
// each thread forms the length-N2 DFTs of its k1 = t + N2 a, ending with X[k1 + N1 k2].
// That output set is again {m : m = t mod N2}, the input distribution, so an inverse can
// start from registers. Small DFTs are radix-2 decimation-in-time with compile-time
// indices; every twiddle comes from the accurate table W (exp(-2 pi i m / N), sincospi).
// The passes move each value once each way with whole 128-byte segments per warp, and no
// integer division is left in the butterflies.
template <int N> struct Split;
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Split<128> { static constexpr int N1 = 16, N2 = 8; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
// exchange buffer of one sequence: N1 rows of N2 + 1 doubles, plus 4 so that consecutive
// sequences' buffers start 8 banks apart
template <int N> constexpr int XchLen = Split<N>::N1 * (Split<N>::N2 + 1) + 4;

__host__ __device__ constexpr int ilog2(int v) { return v >= 16 ? 4 : v >= 8 ? 3 : v >= 4 ? 2 : v >= 2 ? 1 : 0; }
// bit reversal of v in `bits` (<= 4) bits
__host__ __device__ constexpr int bitrev(int v, int bits) {
    const int r4 = ((v & 1) << 3) | ((v & 2) << 1) | ((v & 4) >> 1) | ((v & 8) >> 3);
    return r4 >> (4 - bits);
}

// In-register DFT of length R on (xr, xi) (natural order in and out); w holds W_N^m and
// W_R^j = w[j * (N / R)].
// one radix-2 stage of span M = 2^S over the R registers (compile-time indices)
template <int R, int N, bool INV, int M>
__device__ __forceinline__ void dit_stage(double (&xr)[R], double (&xi)[R], const double2* w) {
    constexpr int H = M / 2;
#pragma unroll
    for (int k = 0; k < R; k += M) {
#pragma unroll
        for (int j = 0; j < H; j++) {
            const double br = xr[k + j + H], bi = xi[k + j + H];
            double tr = br, ti = bi;
            if (j != 0) {
                const double2 tw = w[j * (N / M)];
                const double c = tw.x, sn = INV ? -tw.y : tw.y;
                tr = fma(br, c, -bi * sn);
                ti = fma(br, sn, bi * c);
            }
            const double ur = xr[k + j], ui = xi[k + j];
            xr[k + j] = ur + tr;
            xi[k + j] = ui + ti;
            xr[k + j + H] = ur - tr;
            xi[k + j + H] = ui - ti;
        }
    }
}

template <int R, int N, bool INV>
__device__ __forceinline__ void dft_reg(double (&xr)[R], double (&xi)[R], const double2* w) {
    constexpr int B = ilog2(R);
#pragma unroll
    for (int q = 0; q < R; q++) {  // bit-reversal permutation, in place
        const int p = bitrev(q, B);
        if (q < p) {
            const double tr = xr[q], ti = xi[q];
            xr[q] = xr[p];
            xi[q] = xi[p];
            xr[p] = tr;
            xi[p] = ti;
        }
    }
    dit_stage<R, N, INV, 2>(xr, xi, w);
    dit_stage<R, N, INV, 4>(xr, xi, w);
    dit_stage<R, N, INV, 8>(xr, xi, w);
    if constexpr (R >= 16) dit_stage<R, N, INV, 16>(xr, xi, w);
}

// The distributed length-N transform of one sequence by its N2 threads (t = this thread's
// rank): in, xr[n1] = x[n1 N2 + t]; out, xr[a N2 + k2] = X[(t + N2 a) + N1 k2]. (xre, xim)
// is the sequence's exchange buffer (XchLen<N> doubles each: N1 rows of N2 + 1, the pad
// spreading a warp's accesses over the banks); `sync` makes the writes of all N2 threads
// visible (a warp or block barrier, whichever spans them).
template <int N, bool INV, class Sync>
__device__ __forceinline__ void fft_dist(double (&xr)[Split<N>::N1], double (&xi)[Split<N>::N1], int t,
                                         const double2* w, double* xre, double* xim, Sync sync) {
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    dft_reg<N1, N, INV>(xr, xi, w);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) {
        const double2 tw = w[(t * k1) & (N - 1)];
        const double c = tw.x, sn = INV ? -tw.y : tw.y;
        const double r = xr[k1], i = xi[k1];
        xre[k1 * (N2 + 1) + t] = k1 == 0 ? r : fma(r, c, -i * sn);
        xim[k1 * (N2 + 1) + t] = k1 == 0 ? i : fma(r, sn, i * c);
    }
    sync();
#pragma unroll
    for (int a = 0; a < N1 / N2; a++) {
        double yr[N2], yi[N2];
        const int k1 = t + N2 * a;
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) {
            yr[n2] = xre[k1 * (N2 + 1) + n2];
            yi[n2] = xim[k1 * (N2 + 1) + n2];
        }
        dft_reg<N2, N, INV>(yr, yi, w);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            xr[a * N2 + k2] = yr[k2];
            xi[a * N2 + k2] = yi[k2];
        }
    }
    sync();  // the buffer is free again
}

// Index, in the sequence, of register q after fft_dist (thread t): (t + N2 a) + N1 k2 for
// q = a N2 + k2. It is also the input index n1 N2 + t of register n1 = q' for the inverse:
// X[m] with m = t + N2 n1' sits in register q where n1' = a + (N1 / N2) k2.
template <int N>
__device__ __forceinline__ int out_index(int t, int q) {
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    return (t + N2 * (q / N2)) + N1 * (q % N2);
}

constexpr int kRegRows = 8;  // sequences per CTA in the row and column passes

// pass K forward: real rows of N (q) -> spectrum rows of N/2+1; a CTA of kRegRows x N2
// threads takes kRegRows consecutive rows, thread (r, t) = r N2 + t (a row's threads in one
// warp, reading consecutive values)
template <int N>
__global__ void __launch_bounds__(kRegRows * Split<N>::N2) k_rows_fwd(const double* __restrict__ in,
                                                                    double2* __restrict__ spec,
                                                                    const double2* __restrict__ W, long rows) {
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, NH = N / 2 + 1;
    __shared__ double2 w[N];
    __shared__ double xre[kRegRows][XchLen<N>], xim[kRegRows][XchLen<N>];
    for (int m = threadIdx.x; m < N; m += blockDim.x) w[m] = W[m];
    __syncthreads();
    const int r = threadIdx.x / N2, t = threadIdx.x % N2;
    const long row = (long)blockIdx.x * kRegRows + r;
    const bool live = row < rows;
    double xr[N1], xi[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) {
        xr[n1] = live ? in[row * N + n1 * N2 + t] : 0.0;
        xi[n1] = 0.0;
    }
    fft_dist<N, false>(xr, xi, t, w, xre[r], xim[r], [] { __syncwarp(); });
    if (!live) return;
#pragma unroll
    for (int q = 0; q < N1; q++) {
        const int m = out_index<N>(t, q);
        if (m < NH) spec[row * NH + m] = make_double2(xr[q], xi[q]);
    }
}

// pass K': spectrum rows (Hermitian, N/2+1 stored) -> real rows of N
template <int N>
__global__ void __launch_bounds__(kRegRows * Split<N>::N2) k_rows_inv(const double2* __restrict__ spec,
                                                                    double* __restrict__ out,
                                                                    const double2* __restrict__ W, long rows) {
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, NH = N / 2 + 1;
    __shared__ double2 w[N];
    __shared__ double xre[kRegRows][XchLen<N>], xim[kRegRows][XchLen<N>];
    for (int m = threadIdx.x; m < N; m += blockDim.x) w[m] = W[m];
    __syncthreads();
    const int r = threadIdx.x / N2, t = threadIdx.x % N2;
    const long row = (long)blockIdx.x * kRegRows + r;
    const bool live = row < rows;
    double xr[N1], xi[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) {
        const int m = n1 * N2 + t;
        double2 v = make_double2(0.0, 0.0);
        if (live) {
            if (m < NH) v = spec[row * NH + m];
            else {
                v = spec[row * NH + (N - m)];
                v.y = -v.y;
            }
        }
        xr[n1] = v.x;
        xi[n1] = v.y;
    }
    fft_dist<N, true>(xr, xi, t, w, xre[r], xim[r], [] { __syncwarp(); });
    if (!live) return;
#pragma unroll
    for (int q = 0; q < N1; q++) out[row * N + out_index<N>(t, q)] = xr[q];
}

// passes J / I: columns of the spectrum (MODE 0 forward along j, 1 inverse along j, 2
// forward along i, ig2 multiply, inverse along i). A CTA takes kRegRows consecutive kh of
// one i (MODE 0/1) or one j (MODE 2); thread (t, f) = t kRegRows + f, so a warp reads whole
// 128-byte runs of kh; a column's threads span warps and exchange through the block.
template <int N, int MODE>
__global__ void __launch_bounds__(kRegRows * Split<N>::N2) k_cols_reg(double2* __restrict__ spec,
                                                                    const double2* __restrict__ W,
                                                                    const double* __restrict__ freq,
                                                                    const double* __restrict__ rfreq, double cst) {
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, NH = N / 2 + 1;
    constexpr int NT = (NH + kRegRows - 1) / kRegRows;
    __shared__ double2 w[N];
    __shared__ double xre[kRegRows][XchLen<N>], xim[kRegRows][XchLen<N>];
    for (int m = threadIdx.x; m < N; m += blockDim.x) w[m] = W[m];
    __syncthreads();
    const int t = threadIdx.x / kRegRows, f = threadIdx.x % kRegRows;
    const int fixed = blockIdx.x / NT, kh = (blockIdx.x % NT) * kRegRows + f;
    const bool live = kh < NH;
    const long nnh = (long)N * NH;
    // element e of the column: (i = fixed, j = e) for MODE 0/1, (i = e, j = fixed) for MODE 2
    auto addr = [&](int e) -> long { return MODE == 2 ? (long)e * nnh + (long)fixed * NH + kh
                                                      : (long)fixed * nnh + (long)e * NH + kh; };
    double xr[N1], xi[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) {
        const double2 v = live ? spec[addr(n1 * N2 + t)] : make_double2(0.0, 0.0);
        xr[n1] = v.x;
        xi[n1] = v.y;
    }
    auto bar = [] { __syncthreads(); };
    if (MODE == 1)
        fft_dist<N, true>(xr, xi, t, w, xre[f], xim[f], bar);
    else
        fft_dist<N, false>(xr, xi, t, w, xre[f], xim[f], bar);
    if (MODE == 2) {
        // ig2(i, j, kh) = cst / ((freq_i^2 + freq_j^2) + rfreq_kh^2 + 1e-10), DC untouched
        const double fj = freq[fixed], rk = live ? rfreq[kh] : 0.0;
        double yr[N1], yi[N1];
#pragma unroll
        for (int q = 0; q < N1; q++) {
            const int e = out_index<N>(t, q);
            double g = 1.0;
            if (!(e == 0 && fixed == 0 && kh == 0)) {
                const double fi = freq[e];
                const double f1 = fi * fi;
                const double f2 = f1 + fj * fj;
                g = cst / (f2 + rk * rk + 1E-10);
            }
            // register q holds X[e], e - t = N2 (q / N2) + N1 (q % N2): the inverse's input
            // n1' = (e - t) / N2
            const int n1p = q / N2 + (N1 / N2) * (q % N2);
            yr[n1p] = xr[q] * g;
            yi[n1p] = xi[q] * g;
        }
        fft_dist<N, true>(yr, yi, t, w, xre[f], xim[f], bar);
#pragma unroll
        for (int q = 0; q < N1; q++) {
            xr[q] = yr[q];
            xi[q] = yi[q];
        }
    }
    if (!live) return;
#pragma unroll
    for (int q = 0; q < N1; q++) spec[addr(out_index<N>(t, q))] = make_double2(xr[q], xi[q]);
}

template <int N>
void solve_reg(const double* q, double* phi, double2* spec, const double2* W, const double* freq, const double* rfreq,
               double cst, cudaStream_t s) {
    constexpr int T = kRegRows * Split<N>::N2, NH = N / 2 + 1;
    constexpr int NT = (NH + kRegRows - 1) / kRegRows;
    const long rows = (long)N * N;
    const int rblocks = (int)((rows + kRegRows - 1) / kRegRows);
    count_launch();
    k_rows_fwd<N><<<rblocks, T, 0, s>>>(q, spec, W, rows);
    count_launch();
    k_cols_reg<N, 0><<<N * NT, T, 0, s>>>(spec, W, freq, rfreq, cst);
    count_launch();
    k_cols_reg<N, 2><<<N * NT, T, 0, s>>>(spec, W, freq, rfreq, cst);
    count_launch();
    k_cols_reg<N, 1><<<N * NT, T, 0, s>>>(spec, W, freq, rfreq, cst);
    count_launch();
    k_rows_inv<N><<<rblocks, T, 0, s>>>(spec, phi, W, rows);
    MZB_CHECK(cudaGetLastError());
}

}  // namespace

void FftPoisson::init(int n_, double L_, double h_) {
    release();
    n = n_;
    L = L_;
    h = h_;
    nh = n / 2 + 1;
    (void)plan_radices(n);
    MZB_CHECK(cudaMalloc(&spec, sizeof(double2) * (size_t)n * n * nh));
    MZB_CHECK(cudaMalloc(&W, sizeof(double2) * n));
    MZB_CHECK(cudaMalloc(&freq, sizeof(double) * n));
    MZB_CHECK(cudaMalloc(&rfreq, sizeof(double) * nh));
    count_launch();
    k_twiddles<<<(n + 127) / 128, 128>>>(W, n);
    count_launch();
    k_freqs<<<(n + 127) / 128, 128>>>(freq, rfreq, n, L);
    MZB_CHECK(cudaGetLastError());
    MZB_CHECK(cudaDeviceSynchronize());
    const int rows_smem = (2 * n + 4 * kRowsPerBlock * n) * (int)sizeof(double);
    const int cols_smem = (2 * n + 4 * kColsPerBlock * n) * (int)sizeof(double);
    MZB_CHECK(cudaFuncSetAttribute(k_pass_k_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, rows_smem));
    MZB_CHECK(cudaFuncSetAttribute(k_pass_k_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, rows_smem));
    MZB_CHECK(cudaFuncSetAttribute(k_pass_cols<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, cols_smem));
    MZB_CHECK(cudaFuncSetAttribute(k_pass_cols<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, cols_smem));
    MZB_CHECK(cudaFuncSetAttribute(k_pass_cols<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, cols_smem));
}

void FftPoisson::release() {
    if (spec) cudaFree(spec);
    if (W) cudaFree(W);
    if (freq) cudaFree(freq);
    if (rfreq) cudaFree(rfreq);
    spec = nullptr;
    W = nullptr;
    freq = nullptr;
    rfreq = nullptr;
}

void FftPoisson::solve(const double* q, double* phi, cudaStream_t s) const {
    // constant = 4 pi / (h h h) / (n n n)   (grid_fft.c:105)
    const double cst0 = 4 * kPi / (h * h * h) / (double)(n * n * n);
    if (n == 256) return solve_reg<256>(q, phi, spec, W, freq, rfreq, cst0, s);
    if (n == 128) return solve_reg<128>(q, phi, spec, W, freq, rfreq, cst0, s);
    if (n == 64) return solve_reg<64>(q, phi, spec, W, freq, rfreq, cst0, s);
    const Radices rd = plan_radices(n);
    const long rows = (long)n * n;
    const int rblocks = (int)((rows + kRowsPerBlock - 1) / kRowsPerBlock);
    const int ntk = (nh + kColsPerBlock - 1) / kColsPerBlock;
    const int cblocks = n * ntk;
    const size_t rows_smem = (2 * n + 4 * kRowsPerBlock * n) * sizeof(double);
    const size_t cols_smem = (2 * n + 4 * kColsPerBlock * n) * sizeof(double);
    // constant = 4 pi / (h h h) / (n n n)   (grid_fft.c:105)
    const double cst = 4 * kPi / (h * h * h) / (double)(n * n * n);
    count_launch();
    k_pass_k_fwd<<<rblocks, kFftThreads, rows_smem, s>>>(q, spec, W, n, rd);
    count_launch();
    k_pass_cols<0><<<cblocks, kFftThreads, cols_smem, s>>>(spec, W, n, rd, freq, rfreq, cst);
    count_launch();
    k_pass_cols<2><<<cblocks, kFftThreads, cols_smem, s>>>(spec, W, n, rd, freq, rfreq, cst);
    count_launch();
    k_pass_cols<1><<<cblocks, kFftThreads, cols_smem, s>>>(spec, W, n, rd, freq, rfreq, cst);
    count_launch();
    k_pass_k_inv<<<rblocks, kFftThreads, rows_smem, s>>>(spec, phi, W, n, rd);
    MZB_CHECK(cudaGetLastError());
}

}  // namespace mzb
