// Mixed-radix multi-dimensional FFT of the Toeplitz grids (see grid_fft.cuh).
//
// Stockham autosort, one stage per radix R of the axis length n (Ns = product
// of the radices already applied, T = n / R): butterfly i (k = i mod Ns)
// reads x[i + r T] (r < R), multiplies input r by w_{Ns R}^{r k}, takes the
// R-point DFT and writes output q to y[(i - k) R + k + q Ns].  After the last
// stage y holds the transform in natural order.  The stages alternate between
// two shared-memory buffers, so every stage reads one buffer and writes the
// other with a single barrier in between.
#include "common.cuh"
#include "grid_fft.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

namespace imp {

namespace {

constexpr int kThreads = 256;
constexpr double kPiD = 3.14159265358979323846264338327950288;

// cos / sin of a compile-time angle (|x| <= 2 pi) by Taylor series, folded
// by the compiler into the butterfly constants.
__host__ __device__ constexpr double tsin(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double tcos(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}

__host__ __device__ constexpr int ilog2i(int n) { return n <= 1 ? 0 : 1 + ilog2i(n >> 1); }
__host__ __device__ constexpr int bitrev(int i, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
    return r;
}

// ---- radix 2^m: decimation-in-time network on bit-reversed registers ----
template <int R, int HALF, int K, bool INV>
__device__ __forceinline__ void dit_stage(float2 (&v)[R]) {
    if constexpr (HALF < R) {
        if constexpr (K < HALF) {
            constexpr double ang = -kPiD * K / HALF;
            constexpr float wc = (float)tcos(ang);
            constexpr float ws = (float)(INV ? -tsin(ang) : tsin(ang));
#pragma unroll
            for (int i = 0; i < R; i += 2 * HALF) {
                const float2 a = v[i + K];
                float2 b = v[i + K + HALF];
                if constexpr (K == 0) {
                } else if constexpr (2 * K == HALF) {
                    b = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
                } else {
                    b = make_float2(b.x * wc - b.y * ws, b.x * ws + b.y * wc);
                }
                v[i + K] = make_float2(a.x + b.x, a.y + b.y);
                v[i + K + HALF] = make_float2(a.x - b.x, a.y - b.y);
            }
            dit_stage<R, HALF, K + 1, INV>(v);
        } else {
            dit_stage<R, 2 * HALF, 0, INV>(v);
        }
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft_pow2(float2 (&v)[R]) {
    constexpr int LG = ilog2i(R);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = bitrev(i, LG);
        if (j > i) {
            const float2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
    dit_stage<R, 1, 0, INV>(v);
}

// ---- odd radix: direct R-point DFT with compile-time constants ----
template <int R, bool INV, int K, int Q>
__device__ __forceinline__ void dft_acc(const float2 (&v)[R], float2 &acc) {
    if constexpr (Q < R) {
        constexpr int m = (Q * K) % R;
        if constexpr (m == 0) {
            acc.x += v[Q].x;
            acc.y += v[Q].y;
        } else {
            constexpr double ang = -2.0 * kPiD * m / R;
            constexpr float c = (float)tcos(ang);
            constexpr float s = (float)(INV ? -tsin(ang) : tsin(ang));
            acc.x = fmaf(v[Q].x, c, fmaf(-v[Q].y, s, acc.x));
            acc.y = fmaf(v[Q].x, s, fmaf(v[Q].y, c, acc.y));
        }
        dft_acc<R, INV, K, Q + 1>(v, acc);
    }
}

template <int R, bool INV, int K>
__device__ __forceinline__ void dft_out(const float2 (&v)[R], float2 (&o)[R]) {
    if constexpr (K < R) {
        float2 acc = v[0];
        dft_acc<R, INV, K, 1>(v, acc);
        o[K] = acc;
        dft_out<R, INV, K + 1>(v, o);
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
    if constexpr ((R & (R - 1)) == 0) {
        dft_pow2<R, INV>(v);
    } else {
        float2 o[R];
        dft_out<R, INV, 0>(v, o);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = o[q];
    }
}

__device__ __forceinline__ float2 twid(const float2 *__restrict__ tw, int e, bool inv) {
    float2 w = __ldg(&tw[e]);
    if (inv) w.y = -w.y;
    return w;
}

// Tile geometry of one axis pass: element j of line c of the tile sits at
// c * rs + j + j / 16 of each shared buffer.  The skew (one pad element per 16)
// spreads a stage's stride-R writes over the banks; the row stride rs is
// chosen on the host so that the lines a half-warp touches at once fall on
// different banks too.
struct Tile {
    int n, ln, cw, lcw, rs;
};

__device__ __forceinline__ int sx(const Tile &g, int c, int j) { return c * g.rs + j + (j >> 4); }

// P2: n is a power of two (so is every Ns), index arithmetic by shifts and masks.
template <int R, bool INV, bool P2>
__device__ __forceinline__ void stage(const float2 *__restrict__ A, float2 *__restrict__ B,
                                      const Tile &g, int Ns, const float2 *__restrict__ tw) {
    const int T = g.n / R;
    const int tstep = g.n / (Ns * R);
    const int items = T << g.lcw;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int c = it & (g.cw - 1), i = it >> g.lcw;
        const int k = P2 ? (i & (Ns - 1)) : i % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = A[sx(g, c, i + r * T)];
        if (k) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid(tw, r * k * tstep, INV));
        }
        dft<R, INV>(v);
        const int j0 = (i - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) B[sx(g, c, j0 + q * Ns)] = v[q];
    }
}

// Any radix: each thread computes whole outputs, O(R) work per output.
template <bool INV>
__device__ __forceinline__ void stage_generic(const float2 *__restrict__ A, float2 *__restrict__ B,
                                              const Tile &g, int R, int Ns,
                                              const float2 *__restrict__ tw) {
    const int n = g.n, T = n / R, tstep = n / (Ns * R), rstep = n / R;
    const int items = n << g.lcw;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int c = it & (g.cw - 1), o = it >> g.lcw;
        const int blk = o / (Ns * R), rem = o % (Ns * R);
        const int q = rem / Ns, k = rem % Ns;
        const int i = blk * Ns + k;
        const int step = k * tstep + q * rstep;
        float2 acc = make_float2(0.f, 0.f);
        int e = 0;
        for (int r = 0; r < R; ++r) {
            const float2 u = cmul(A[sx(g, c, i + r * T)], twid(tw, e, INV));
            acc.x += u.x;
            acc.y += u.y;
            e += step;
            if (e >= n) e -= n * (e / n);
        }
        B[sx(g, c, o)] = acc;
    }
}

struct AxisArgs {
    long long S;       // element stride of the axis (product of the faster lengths)
    int n, ln;         // axis length and its log2 (when a power of two)
    int cw, lcw, rs;   // lines per block (power of two), log2(cw), tile row stride
    int nst;           // stages
    unsigned char rad[24];
    // Pruning.  Outputs kept along this axis: j < klo or j >= n - khi (klo = n:
    // all).  Lines: only those whose coordinates along the faster axes are kept
    // there, enumerated compactly: nf faster axes (outer first) with kept
    // ranges [0, flo) and [fg - fhi, fg); Sc = product of their kept counts.
    int klo, khi;
    int nf;
    int flo[2], fhi[2], fg[2];
    long long Sc;
};

// Offset (within S) of compact line index ic over the kept faster coordinates.
__device__ __forceinline__ long long line_offset(const AxisArgs &p, long long ic) {
    auto ex = [](long long c, int lo, int hi, int g) -> long long {
        return c < lo ? c : c + (g - lo - hi);
    };
    if (p.nf == 0) return ic;
    if (p.nf == 1) return ex(ic, p.flo[0], p.fhi[0], p.fg[0]);
    const long long inner = p.flo[1] + p.fhi[1];
    const long long y = ic / inner, z = ic - y * inner;
    return ex(y, p.flo[0], p.fhi[0], p.fg[0]) * p.fg[1] + ex(z, p.flo[1], p.fhi[1], p.fg[1]);
}

constexpr int kLoadUnroll = 4;  // global loads a thread issues before its shared stores

// One axis pass.  Block b takes lines l0 = b cw .. l0 + cw - 1 (line l = o S + i
// starts at o n S + i): consecutive columns of a strided axis (cw divides S),
// consecutive whole lines of the contiguous one (S = 1).
template <bool INV, bool P2>
__global__ void __launch_bounds__(kThreads) k_fft_axis(float2 *__restrict__ data, AxisArgs p,
                                                       const float2 *__restrict__ tw) {
    extern __shared__ float2 sm[];
    const int n = p.n;
    const bool contig = p.S == 1;
    Tile g;
    g.n = n;
    g.ln = p.ln;
    g.cw = p.cw;
    g.lcw = p.lcw;
    g.rs = p.rs;
    float2 *A = sm, *B = sm + p.cw * p.rs;
    const long long l0 = (long long)blockIdx.x * p.cw;
    const int E = n << p.lcw;
    const int step = blockDim.x * kLoadUnroll;
    // line and element of flat tile index e (contiguous: line-major; strided: column-major)
    auto split = [&](int e, int &c, int &j) {
        if (contig) {
            c = P2 ? e >> p.ln : e / n;
            j = e - c * n;
        } else {
            c = e & (p.cw - 1);
            j = e >> p.lcw;
        }
    };
    // strided: the block's lines are compact indices l0 .. l0 + cw - 1 over (slower
    // coordinate o, kept faster coordinates); cw divides the innermost kept range
    const long long o = contig ? 0 : l0 / p.Sc;
    const long long i0 = contig ? 0 : line_offset(p, l0 - o * p.Sc);
    float2 *base = contig ? data + l0 * n : data + o * n * p.S + i0;
    auto gaddr = [&](int e, int c, int j) -> long long {
        return contig ? (long long)e : (long long)j * p.S + c;
    };
    for (int e0 = threadIdx.x; e0 < E; e0 += step) {
        float2 v[kLoadUnroll];
#pragma unroll
        for (int u = 0; u < kLoadUnroll; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < E) {
                int c, j;
                split(e, c, j);
                v[u] = base[gaddr(e, c, j)];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadUnroll; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < E) {
                int c, j;
                split(e, c, j);
                A[sx(g, c, j)] = v[u];
            }
        }
    }
    __syncthreads();
    int Ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.rad[s];
        switch (R) {
            case 2: stage<2, INV, P2>(A, B, g, Ns, tw); break;
            case 3: stage<3, INV, P2>(A, B, g, Ns, tw); break;
            case 4: stage<4, INV, P2>(A, B, g, Ns, tw); break;
            case 5: stage<5, INV, P2>(A, B, g, Ns, tw); break;
            case 7: stage<7, INV, P2>(A, B, g, Ns, tw); break;
            case 8: stage<8, INV, P2>(A, B, g, Ns, tw); break;
            case 16: stage<16, INV, P2>(A, B, g, Ns, tw); break;
            default: stage_generic<INV>(A, B, g, R, Ns, tw); break;
        }
        __syncthreads();
        float2 *t = A;
        A = B;
        B = t;
        Ns *= R;
    }
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        int c, j;
        split(e, c, j);
        if (j >= p.klo && j < n - p.khi) continue;  // output cropped away
        base[gaddr(e, c, j)] = A[sx(g, c, j)];
    }
}

// Tile row stride for lines of n points, cw lines per block: long enough for
// the skewed line, and such that the rows a half-warp touches at once (16 / cw
// elements of each of cw lines, or 16 lines) start on distinct bank pairs.
int row_stride(int n, int cw) {
    const int base = n + ((n - 1) >> 4);
    const int m = cw >= 16 ? 2 : 32 / cw, t = cw >= 16 ? 1 : 16 / cw;
    int rs = base;
    while (rs % m != t % m) ++rs;
    return rs;
}

// Radices of n: 16s, then 8, 4, 2, then 3, 5, 7, then any other prime.
int factorize(int n, unsigned char *out) {
    int k = 0;
    for (int r : {16, 8, 4, 2})
        while (n % r == 0) {
            out[k++] = (unsigned char)r;
            n /= r;
        }
    for (int r : {3, 5, 7})
        while (n % r == 0) {
            out[k++] = (unsigned char)r;
            n /= r;
        }
    for (int p = 11; n > 1; p += 2)
        while (n % p == 0) {
            out[k++] = (unsigned char)p;  // p <= kGridFftMaxN: values above 255 are refused
            n /= p;
        }
    return k;
}

// True when every prime factor of n fits the radix table (<= 255).
bool radices_fit(int n) {
    for (int p = 2; n > 1; ++p) {
        if (n % p) continue;
        if (p > 255) return false;
        while (n % p == 0) n /= p;
    }
    return true;
}

int pow2_divisor_le(long long v, int cap) {
    int c = 1;
    while (c * 2 <= cap && v % (c * 2) == 0) c *= 2;
    return c;
}

}  // namespace

cudaError_t grid_fft_create(GridFft *f, int n0, int n1, int n2, int batch) {
    grid_fft_destroy(f);
    const int n[3] = {n0, n1, n2};
    for (int a = 0; a < 3; ++a) {
        if (n[a] < 1 || n[a] > kGridFftMaxN || !radices_fit(n[a])) return cudaErrorInvalidValue;
        f->n[a] = n[a];
    }
    if (batch < 1) return cudaErrorInvalidValue;
    f->batch = batch;
    {  // per device: set on every plan (cheap)
        const int lim = 160 * 1024;
        cudaError_t e = cudaSuccess;
        for (const void *k : {(const void *)k_fft_axis<false, false>,
                              (const void *)k_fft_axis<true, false>,
                              (const void *)k_fft_axis<false, true>,
                              (const void *)k_fft_axis<true, true>})
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        if (e != cudaSuccess) return e;
    }
    for (int a = 0; a < 3; ++a) {
        const int len = n[a];
        if (len == 1) continue;
        f->nfac[a] = factorize(len, f->fac[a]);
        long long S = 1, O = batch;
        for (int b = a + 1; b < 3; ++b) S *= n[b];
        for (int b = 0; b < a; ++b) O *= n[b];
        int cw;
        if (S == 1) {
            cw = pow2_divisor_le(O, std::max(1, std::min(64, 4096 / len)));
        } else {
            int cap = std::max(1, std::min(32, 4096 / len));
            if (cap < 4) cap = std::max(1, std::min(4, 8192 / len));
            cw = pow2_divisor_le(S, cap);
        }
        f->cw[a] = cw;
        f->rs[a] = row_stride(len, cw);
        f->smem[a] = sizeof(float2) * 2 * (size_t)cw * f->rs[a];
        std::vector<float2> h(len);
        for (int j = 0; j < len; ++j) {
            const double ang = -2.0 * kPiD * (double)j / (double)len;
            h[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        cudaError_t e = cudaMalloc(&f->tw[a], sizeof(float2) * len);
        if (e == cudaSuccess)
            e = cudaMemcpy(f->tw[a], h.data(), sizeof(float2) * len, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            grid_fft_destroy(f);
            return e;
        }
    }
    return cudaSuccess;
}

void grid_fft_destroy(GridFft *f) {
    for (int a = 0; a < 3; ++a) {
        if (f->tw[a]) cudaFree(f->tw[a]);
        f->tw[a] = nullptr;
    }
}

cudaError_t grid_fft_exec(const GridFft &f, float2 *data, bool inverse, cudaStream_t st) {
    return grid_fft_exec_cropped(f, data, inverse, nullptr, st);
}

cudaError_t grid_fft_exec_cropped(const GridFft &f, float2 *data, bool inverse,
                                  const int keep_half[3], cudaStream_t st) {
    // kept output range per axis: [0, lo) and [n - hi, n)
    int klo[3], khi[3];
    for (int a = 0; a < 3; ++a) {
        const int h = keep_half ? keep_half[a] : 0;
        if (h > 0 && 2 * h <= f.n[a]) {
            klo[a] = h;
            khi[a] = h;
        } else {
            klo[a] = f.n[a];
            khi[a] = 0;
        }
    }
    // the fastest axis first: its pass is the one whose reads and writes are
    // whole contiguous lines; later passes only take lines kept by earlier ones
    for (int a = 2; a >= 0; --a) {
        const int len = f.n[a];
        if (len == 1) continue;
        AxisArgs p;
        p.S = 1;
        long long O = f.batch;
        for (int b = a + 1; b < 3; ++b) p.S *= f.n[b];
        for (int b = 0; b < a; ++b) O *= f.n[b];
        p.n = len;
        p.ln = ilog2i(len);
        p.nst = f.nfac[a];
        for (int s = 0; s < p.nst; ++s) p.rad[s] = f.fac[a][s];
        p.klo = klo[a];
        p.khi = khi[a];
        p.nf = 0;
        p.Sc = 1;
        int inner_lo = 0, inner_hi = 0;
        bool gap = false;
        for (int b = a + 1; b < 3; ++b) {
            if (f.n[b] == 1) continue;
            p.flo[p.nf] = klo[b];
            p.fhi[p.nf] = khi[b];
            p.fg[p.nf] = f.n[b];
            p.Sc *= (long long)(klo[b] + khi[b]);
            inner_lo = klo[b];
            inner_hi = khi[b];
            gap = gap || khi[b] > 0;
            ++p.nf;
        }
        p.cw = f.cw[a];
        if (p.S > 1 && gap) {  // a block's columns must be consecutive in memory
            while (p.cw > 1 && (p.Sc % p.cw || inner_lo % p.cw || inner_hi % p.cw)) p.cw >>= 1;
        }
        p.lcw = ilog2i(p.cw);
        p.rs = row_stride(len, p.cw);
        const size_t smem = sizeof(float2) * 2 * (size_t)p.cw * p.rs;
        const long long blocks = (p.S > 1 ? O * p.Sc : O) / p.cw;
        if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
        const bool p2 = (len & (len - 1)) == 0;
        const unsigned nb = (unsigned)blocks;
        if (inverse) {
            if (p2) k_fft_axis<true, true><<<nb, kThreads, smem, st>>>(data, p, f.tw[a]);
            else k_fft_axis<true, false><<<nb, kThreads, smem, st>>>(data, p, f.tw[a]);
        } else {
            if (p2) k_fft_axis<false, true><<<nb, kThreads, smem, st>>>(data, p, f.tw[a]);
            else k_fft_axis<false, false><<<nb, kThreads, smem, st>>>(data, p, f.tw[a]);
        }
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace imp
