// elliptic.cu -- multi-domain Poisson / Helmholtz solves by DST-I on B200.
//
// Replaces the reference's EllipticSolver::solve (src/EllipticSolver.cc:47-73)
// and EllipticSolver2d (src/EllipticSolver2d.cc:26-185): each level is solved
// with zero or lifted boundary values by a 2-D DST-I (FFTW RODFT00), a
// diagonal eigenvalue scaling and an inverse DST-I, coarse levels first.
//
// Design (one level, nodes NI x NJ, j contiguous):
//   pass A  rows:    load rhs (+ boundary lifting from the coarser solution),
//                    DST-I along j                          -> T
//   pass B  columns: DST-I along i, x eigen-inverse, DST-I   -> T (in place)
//   pass C  rows:    DST-I along j, x 1/(4 nx ny)            -> u (+ base - u)
// A DST-I of length n is read off the DFT of the odd extension of length
// m = 2(n+1).  Two real lines a, b are packed as z = a + i b: the DFT of an
// odd real sequence is purely imaginary, so DST(a)_k = -Im Z_{k+1} and
// DST(b)_k = Re Z_{k+1}.  The complex FFT is a shared-memory Stockham
// autosort FFT with mixed radices; twiddles are tabulated on the host.
#include "ibg_internal.cuh"
#include "ibg_kernels.cuh"

namespace ibg {

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

template <typename C> __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) { C r; r.x = a; r.y = b; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// one radix-R Stockham butterfly
template <typename C, int R>
__device__ __forceinline__ void bfly(const C* __restrict__ sp, C* __restrict__ dp, const C* __restrict__ tw,
                                     int m, int mr, int ns, int tstep, int j) {
    const int jm = j % ns;
    C v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        C x = sp[j + q * mr];
        v[q] = q == 0 ? x : cmul(x, tw[jm * q * tstep]);
    }
    C o[R];
    if (R == 2) {
        o[0] = cadd(v[0], v[1]);
        o[1] = csub(v[0], v[1]);
    } else if (R == 4) {
        C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        C t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
        o[0] = cadd(t0, t2);
        o[2] = csub(t0, t2);
        o[1] = cmk<C>(t1.x + t3.y, t1.y - t3.x);  // t1 - i t3
        o[3] = cmk<C>(t1.x - t3.y, t1.y + t3.x);  // t1 + i t3
    } else {
        const int rstep = m / R;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            C acc = v[0];
#pragma unroll
            for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], tw[((k * q) % R) * rstep]));
            o[k] = acc;
        }
    }
    const int idxd = (j / ns) * ns * R + jm;
#pragma unroll
    for (int k = 0; k < R; ++k) dp[idxd + k * ns] = o[k];
}

// generic radix (R <= kMaxRadix) for odd prime factors above 5
template <typename C>
__device__ void bfly_generic(const C* __restrict__ sp, C* __restrict__ dp, const C* __restrict__ tw,
                             int R, int m, int mr, int ns, int tstep, int j) {
    const int jm = j % ns;
    const int rstep = m / R;
    const int idxd = (j / ns) * ns * R + jm;
    for (int k = 0; k < R; ++k) {
        C acc = sp[j];
        for (int q = 1; q < R; ++q) {
            C x = cmul(sp[j + q * mr], tw[jm * q * tstep]);
            acc = cadd(acc, cmul(x, tw[((k * q) % R) * rstep]));
        }
        dp[idxd + k * ns] = acc;
    }
}

// P complex FFTs of length d.m held in s0 (P*m each); returns the buffer holding the result.
template <typename C>
__device__ C* fft_smem(C* s0, C* s1, const C* tw, const FftDesc& d, int P) {
    const int m = d.m;
    int ns = 1;
    C* src = s0;
    C* dst = s1;
    for (int s = 0; s < d.nfac; ++s) {
        const int R = d.fac[s];
        const int mr = m / R;
        const int tstep = m / (ns * R);
        const int total = P * mr;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            const int p = t / mr;
            const int j = t - p * mr;
            const C* sp = src + p * m;
            C* dp = dst + p * m;
            switch (R) {
                case 2: bfly<C, 2>(sp, dp, tw, m, mr, ns, tstep, j); break;
                case 3: bfly<C, 3>(sp, dp, tw, m, mr, ns, tstep, j); break;
                case 4: bfly<C, 4>(sp, dp, tw, m, mr, ns, tstep, j); break;
                case 5: bfly<C, 5>(sp, dp, tw, m, mr, ns, tstep, j); break;
                default: bfly_generic<C>(sp, dp, tw, R, m, mr, ns, tstep, j); break;
            }
        }
        __syncthreads();
        C* t = src; src = dst; dst = t;
        ns *= R;
    }
    return src;
}

template <typename C>
__device__ __forceinline__ void load_twiddles(C* tws, const FftDesc& d) {
    const C* g = reinterpret_cast<const C*>(d.tw);
    for (int k = threadIdx.x; k < d.m; k += blockDim.x) tws[k] = g[k];
}

// ---------------------------------------------------------------------------
// pass A / pass C: transforms along j for pairs of rows
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_dst_rows(RowPassArgs<T> a) {
    using C = typename Cplx<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const FftDesc& d = a.fft;
    const int m = d.m;
    const int P = a.pairs_per_block;
    C* tws = reinterpret_cast<C*>(smem_raw);
    C* s0 = tws + m;
    C* s1 = s0 + P * m;
    const GridDev& g = a.g;
    const int n = g.NJ;
    const size_t ioff = (size_t)blockIdx.y * a.in_bstride;
    const size_t ooff = (size_t)blockIdx.y * a.out_bstride;
    const T* in = a.in + ioff;
    const T* coarse = a.coarse ? a.coarse + ioff : nullptr;
    const int pair0 = blockIdx.x * P;
    const int npairs = (g.NI + 1) / 2;
    load_twiddles(tws, d);
    // fill the odd extensions
    for (int t = threadIdx.x; t < P * n; t += blockDim.x) {
        const int p = t / n;
        const int k = t - p * n;
        const int pair = pair0 + p;
        C* z = s0 + p * m;
        T va = (T)0, vb = (T)0;
        if (pair < npairs) {
            const int r0 = 2 * pair, r1 = 2 * pair + 1;
            va = in[(size_t)r0 * n + k];
            if (r1 < g.NI) vb = in[(size_t)r1 * n + k];
            if (a.lift) {
                // input scale and boundary lifting (getRHS, src/EllipticSolver2d.cc:125-144, :166-185)
                va = a.in_scale * va;
                vb = a.in_scale * vb;
                if (coarse) {
                    const T c = a.bc_coef;
                    const int I0 = r0 + 1, I1 = r1 + 1, J = k + 1;
                    if (k == 0) {
                        va = va - bc_bottom(coarse, g, I0) * c;
                        if (r1 < g.NI) vb = vb - bc_bottom(coarse, g, I1) * c;
                    }
                    if (k == n - 1) {
                        va = va - bc_top(coarse, g, I0) * c;
                        if (r1 < g.NI) vb = vb - bc_top(coarse, g, I1) * c;
                    }
                    if (I0 == 1) va = va - bc_left(coarse, g, J) * c;
                    if (I0 == g.nx - 1) va = va - bc_right(coarse, g, J) * c;
                    if (r1 < g.NI) {
                        if (I1 == g.nx - 1) vb = vb - bc_right(coarse, g, J) * c;
                    }
                }
            }
        }
        z[k + 1] = cmk<C>(va, vb);
        z[m - 1 - k] = cmk<C>(-va, -vb);
        if (k == 0) {
            z[0] = cmk<C>((T)0, (T)0);
            z[n + 1] = cmk<C>((T)0, (T)0);
        }
    }
    __syncthreads();
    C* res = fft_smem<C>(s0, s1, tws, d, P);
    // write out
    T* out = a.out + ooff;
    T* out2 = a.out2 ? a.out2 + ooff : nullptr;
    const T* base = a.base ? a.base + ooff : nullptr;
    for (int t = threadIdx.x; t < P * n; t += blockDim.x) {
        const int p = t / n;
        const int k = t - p * n;
        const int pair = pair0 + p;
        if (pair >= npairs) continue;
        const C z = res[p * m + k + 1];
        const int r0 = 2 * pair, r1 = 2 * pair + 1;
        const size_t i0 = (size_t)r0 * n + k;
        T va = -z.y, vb = z.x;
        if (a.norm != (T)1) { va = va * a.norm; vb = vb * a.norm; }
        out[i0] = va;
        if (out2) out2[i0] = base[i0] - va;
        if (r1 < g.NI) {
            const size_t i1 = (size_t)r1 * n + k;
            out[i1] = vb;
            if (out2) out2[i1] = base[i1] - vb;
        }
    }
}

// ---------------------------------------------------------------------------
// pass B: transforms along i for pairs of columns, eigen-inverse scaling,
// inverse transform along i (in place on T)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_dst_cols(ColPassArgs<T> a) {
    using C = typename Cplx<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const FftDesc& d = a.fft;
    const int m = d.m;
    const int P = a.pairs_per_block;
    C* tws = reinterpret_cast<C*>(smem_raw);
    C* s0 = tws + m;
    C* s1 = s0 + P * m;
    const GridDev& g = a.g;
    const int n = g.NI;
    const int NJ = g.NJ;
    T* buf = a.buf + (size_t)blockIdx.y * a.bstride;
    const int col0 = blockIdx.x * 2 * P;
    const int w = 2 * P;
    load_twiddles(tws, d);
    for (int t = threadIdx.x; t < n * w; t += blockDim.x) {
        const int i = t / w;
        const int c = t - i * w;
        const int col = col0 + c;
        const T v = col < NJ ? buf[(size_t)i * NJ + col] : (T)0;
        C* z = s0 + (c >> 1) * m;
        if (c & 1) {
            z[i + 1].y = v;
            z[m - 1 - i].y = -v;
        } else {
            z[i + 1].x = v;
            z[m - 1 - i].x = -v;
        }
    }
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        s0[p * m] = cmk<C>((T)0, (T)0);
        s0[p * m + n + 1] = cmk<C>((T)0, (T)0);
    }
    __syncthreads();
    C* res = fft_smem<C>(s0, s1, tws, d, P);
    C* other = (res == s0) ? s1 : s0;
    // eigen-inverse scaling; build the second odd extension in `other`
    const T* cx = a.cosx;
    const T* cy = a.cosy;
    for (int t = threadIdx.x; t < P * n; t += blockDim.x) {
        const int p = t / n;
        const int k = t - p * n;
        const C z = res[p * m + k + 1];
        const int ca = col0 + 2 * p, cb = ca + 1;
        T va = -z.y, vb = z.x;
        // lambda_ij = 2 (cos(pi i/nx) + cos(pi j/ny) - 2) / dx^2  (src/EllipticSolver2d.cc:42-54)
        const T ex = cx[k + 1];
        const T la = (T)2 * (ex + cy[(ca < NJ ? ca : 0) + 1] - (T)2) * a.bydx2;
        const T lb = (T)2 * (ex + cy[(cb < NJ ? cb : 0) + 1] - (T)2) * a.bydx2;
        const T ea = a.helmholtz ? (T)1 / ((T)1 + a.alpha * la) : (T)1 / la;
        const T eb = a.helmholtz ? (T)1 / ((T)1 + a.alpha * lb) : (T)1 / lb;
        va = va * ea;
        vb = vb * eb;
        C* zo = other + p * m;
        zo[k + 1] = cmk<C>(va, vb);
        zo[m - 1 - k] = cmk<C>(-va, -vb);
        if (k == 0) {
            zo[0] = cmk<C>((T)0, (T)0);
            zo[n + 1] = cmk<C>((T)0, (T)0);
        }
    }
    __syncthreads();
    C* res2 = fft_smem<C>(other, res, tws, d, P);
    for (int t = threadIdx.x; t < n * w; t += blockDim.x) {
        const int i = t / w;
        const int c = t - i * w;
        const int col = col0 + c;
        if (col >= NJ) continue;
        const C z = res2[(c >> 1) * m + i + 1];
        buf[(size_t)i * NJ + col] = (c & 1) ? z.x : -z.y;
    }
}

// ---------------------------------------------------------------------------
// coarsify one level (src/Scalar.cc:46-64): dst[lev] = f[lev] outside the
// overlap, full-weighting of src (= level lev-1 already coarsified) inside.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_coarsify(GridDev g, const T* f_lev, const T* src_fine, T* dst_lev, size_t bstride) {
    const size_t boff = (size_t)blockIdx.y * bstride;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.N1) return;
    const int i = idx / g.NJ + 1;
    const int j = idx % g.NJ + 1;
    const T* sf = src_fine + boff;
    T v;
    if (i > g.nxe && i < g.nx / 2 + g.nxe && j > g.nye && j < g.ny / 2 + g.nye) {
        const int ii = (i - g.nxe) * 2, jj = (j - g.nye) * 2;
        v = (T)0.25 * node(sf, g, ii, jj) +
            (T)0.125 * (node(sf, g, ii + 1, jj) + node(sf, g, ii, jj + 1) + node(sf, g, ii - 1, jj) +
                        node(sf, g, ii, jj - 1)) +
            (T)0.0625 * (node(sf, g, ii + 1, jj + 1) + node(sf, g, ii + 1, jj - 1) + node(sf, g, ii - 1, jj + 1) +
                         node(sf, g, ii - 1, jj - 1));
    } else {
        v = f_lev[boff + idx];
    }
    dst_lev[boff + idx] = v;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static void factorize(int m, FftDesc& d) {
    d.m = m;
    d.nfac = 0;
    int n = m;
    const int pref[4] = {4, 2, 3, 5};
    for (int r : pref)
        while (n % r == 0 && d.nfac < kMaxFactors) { d.fac[d.nfac++] = r; n /= r; }
    for (int r = 7; n > 1 && d.nfac < kMaxFactors; r += 2)
        while (n % r == 0) { d.fac[d.nfac++] = r; n /= r; }
    if (n != 1) d.nfac = -1;
}

void fft_describe(int m, FftDesc& d) { factorize(m, d); }

bool fft_supported(int m) {
    FftDesc d;
    factorize(m, d);
    if (d.nfac < 0) return false;
    for (int s = 0; s < d.nfac; ++s)
        if (d.fac[s] > kMaxRadix) return false;
    return true;
}

int FftTables::init(int m_rows, int m_cols) {
    factorize(m_rows, row64);
    factorize(m_cols, col64);
    if (!fft_supported(m_rows) || !fft_supported(m_cols)) return IBG_ERR_UNSUPPORTED;
    row32 = row64;
    col32 = col64;
    const double pi = 3.14159265358979323846264338327950288;
    auto make = [&](int m, void** d64, void** d32) -> int {
        std::vector<double2> h64(m);
        std::vector<float2> h32(m);
        for (int k = 0; k < m; ++k) {
            double ang = -2.0 * pi * (double)k / (double)m;
            h64[k] = make_double2(cos(ang), sin(ang));
            h32[k] = make_float2((float)h64[k].x, (float)h64[k].y);
        }
        if (cudaMalloc(d64, sizeof(double2) * m) != cudaSuccess) return IBG_ERR_CUDA;
        if (cudaMalloc(d32, sizeof(float2) * m) != cudaSuccess) return IBG_ERR_CUDA;
        cudaMemcpy(*d64, h64.data(), sizeof(double2) * m, cudaMemcpyHostToDevice);
        cudaMemcpy(*d32, h32.data(), sizeof(float2) * m, cudaMemcpyHostToDevice);
        return IBG_OK;
    };
    int st = make(m_rows, &tw_row64, &tw_row32);
    if (st) return st;
    st = make(m_cols, &tw_col64, &tw_col32);
    if (st) return st;
    row64.tw = tw_row64;
    col64.tw = tw_col64;
    row32.tw = tw_row32;
    col32.tw = tw_col32;
    return IBG_OK;
}

void FftTables::release() {
    cudaFree(tw_row64); cudaFree(tw_row32); cudaFree(tw_col64); cudaFree(tw_col32);
    tw_row64 = tw_row32 = tw_col64 = tw_col32 = nullptr;
}

template <typename T>
static int rows_pairs_per_block(int m) {
    // keep the FFT working set near 64 KB and the grid large
    int budget = (int)(65536 / (2 * sizeof(T) * 2));
    int P = budget / m;
    if (P < 1) P = 1;
    if (P > 4) P = 4;
    return P;
}

template <typename T>
size_t fft_smem_bytes(int m, int P) {
    return sizeof(typename Cplx<T>::type) * (size_t)m * (2 * P + 1);
}

template <typename T>
int EllipticPlan<T>::solve(const SolveCall<T>& c, cudaStream_t st) const {
    const GridDev& g = *grid;
    const int L = g.L;
    const size_t N1 = g.N1;
    const int batch = c.batch;
    if (batch < 1 || batch > 65535) return IBG_ERR_ARG;
    // 1. coarsify the right-hand side into rc (levels 1..L-1)
    for (int lev = 1; lev < L; ++lev) {
        const T* src = (lev == 1) ? c.f : c.rc + (size_t)(lev - 1) * N1;
        dim3 grd((unsigned)((N1 + 255) / 256), (unsigned)batch);
        k_coarsify<T><<<grd, 256, 0, st>>>(g, c.f + (size_t)lev * N1, src, c.rc + (size_t)lev * N1, c.bstride);
    }
    const FftDesc& frow = sizeof(T) == 8 ? tables->row64 : tables->row32;
    const FftDesc& fcol = sizeof(T) == 8 ? tables->col64 : tables->col32;
    const int Pr = rows_pairs;
    const int Pc = cols_pairs;
    const size_t smr = fft_smem_bytes<T>(frow.m, Pr);
    const size_t smc = fft_smem_bytes<T>(fcol.m, Pc);
    const int npairs_r = (g.NI + 1) / 2;
    const int ncolblk = (g.NJ + 2 * Pc - 1) / (2 * Pc);
    // 2. coarse-to-fine sweep
    for (int lev = L - 1; lev >= 0; --lev) {
        const double dxl = lev_dx(g, lev);
        const T* rhs = (lev == 0) ? c.f : c.rc + (size_t)lev * N1;
        RowPassArgs<T> A{};
        A.g = g;
        A.fft = frow;
        A.pairs_per_block = Pr;
        A.in = rhs;
        A.out = c.tbuf;
        A.in_bstride = c.bstride;
        A.out_bstride = N1;
        A.lift = 1;
        A.in_scale = c.in_scale;
        A.coarse = (lev == L - 1) ? nullptr : c.u + (size_t)(lev + 1) * N1;
        A.bc_coef = helmholtz ? (T)(alpha / (dxl * dxl)) : (T)(1.0 / (dxl * dxl));
        A.norm = (T)1;
        k_dst_rows<T><<<dim3((unsigned)((npairs_r + Pr - 1) / Pr), (unsigned)batch), threads, smr, st>>>(A);
        ColPassArgs<T> B{};
        B.g = g;
        B.fft = fcol;
        B.pairs_per_block = Pc;
        B.buf = c.tbuf;
        B.bstride = N1;
        B.cosx = (const T*)(sizeof(T) == 8 ? (const void*)cos64x : (const void*)cos32x);
        B.cosy = (const T*)(sizeof(T) == 8 ? (const void*)cos64y : (const void*)cos32y);
        B.bydx2 = (T)(1.0 / (dxl * dxl));
        B.helmholtz = helmholtz;
        B.alpha = (T)alpha;
        k_dst_cols<T><<<dim3((unsigned)ncolblk, (unsigned)batch), threads, smc, st>>>(B);
        RowPassArgs<T> Cc{};
        Cc.g = g;
        Cc.fft = frow;
        Cc.pairs_per_block = Pr;
        Cc.in = c.tbuf;
        Cc.out = c.u + (size_t)lev * N1;
        Cc.in_bstride = N1;
        Cc.out_bstride = c.bstride;
        Cc.lift = 0;
        Cc.in_scale = (T)1;
        Cc.coarse = nullptr;
        Cc.norm = (T)(1.0 / (double)(2 * g.nx * 2 * g.ny));
        Cc.out2 = c.out2 ? c.out2 + (size_t)lev * N1 : nullptr;
        Cc.base = c.base ? c.base + (size_t)lev * N1 : nullptr;
        k_dst_rows<T><<<dim3((unsigned)((npairs_r + Pr - 1) / Pr), (unsigned)batch), threads, smr, st>>>(Cc);
    }
    return cudaPeekAtLastError() == cudaSuccess ? IBG_OK : IBG_ERR_CUDA;
}

template <typename T>
void EllipticPlan<T>::run_pass(int which, const T* in, T* tbuf, cudaStream_t st) const {
    const GridDev& g = *grid;
    const FftDesc& frow = sizeof(T) == 8 ? tables->row64 : tables->row32;
    const FftDesc& fcol = sizeof(T) == 8 ? tables->col64 : tables->col32;
    const int Pr = rows_pairs, Pc = cols_pairs;
    if (which == 0) {
        RowPassArgs<T> A{};
        A.g = g; A.fft = frow; A.pairs_per_block = Pr; A.in = in; A.out = tbuf;
        A.in_bstride = g.N1; A.out_bstride = g.N1; A.lift = 1; A.in_scale = (T)1; A.coarse = nullptr;
        A.norm = (T)1;
        const int npairs_r = (g.NI + 1) / 2;
        k_dst_rows<T><<<dim3((unsigned)((npairs_r + Pr - 1) / Pr), 1), threads, fft_smem_bytes<T>(frow.m, Pr), st>>>(A);
    } else {
        ColPassArgs<T> B{};
        B.g = g; B.fft = fcol; B.pairs_per_block = Pc; B.buf = tbuf; B.bstride = g.N1;
        B.cosx = (const T*)(sizeof(T) == 8 ? (const void*)cos64x : (const void*)cos32x);
        B.cosy = (const T*)(sizeof(T) == 8 ? (const void*)cos64y : (const void*)cos32y);
        B.bydx2 = (T)(1.0 / (g.dx * g.dx)); B.helmholtz = helmholtz; B.alpha = (T)alpha;
        const int ncolblk = (g.NJ + 2 * Pc - 1) / (2 * Pc);
        k_dst_cols<T><<<dim3((unsigned)ncolblk, 1), threads, fft_smem_bytes<T>(fcol.m, Pc), st>>>(B);
    }
}

template <typename T>
int EllipticPlan<T>::init(const GridDev* g, const FftTables* t, bool helm, double a, const CosTables& ct) {
    grid = g;
    tables = t;
    helmholtz = helm ? 1 : 0;
    alpha = a;
    cos64x = ct.x64; cos64y = ct.y64; cos32x = ct.x32; cos32y = ct.y32;
    const FftDesc& frow = sizeof(T) == 8 ? t->row64 : t->row32;
    const FftDesc& fcol = sizeof(T) == 8 ? t->col64 : t->col32;
    rows_pairs = rows_pairs_per_block<T>(frow.m);
    cols_pairs = rows_pairs_per_block<T>(fcol.m);
    // enough blocks to cover the SMs: at these sizes one or two pairs per block
    if ((g->NI + 1) / 2 / rows_pairs < 296) rows_pairs = 1;
    if (g->NJ / (2 * cols_pairs) < 296) cols_pairs = 1;
    threads = 128;
    size_t smr = fft_smem_bytes<T>(frow.m, rows_pairs);
    size_t smc = fft_smem_bytes<T>(fcol.m, cols_pairs);
    if (smr > 227 * 1024 || smc > 227 * 1024) return IBG_ERR_UNSUPPORTED;
    if (cudaFuncSetAttribute(k_dst_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess)
        return IBG_ERR_CUDA;
    if (cudaFuncSetAttribute(k_dst_cols<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess)
        return IBG_ERR_CUDA;
    return IBG_OK;
}

int CosTables::init(int nx, int ny) {
    // cos(pi i / nx), i = 0..nx-1 and cos(pi j / ny), j = 0..ny-1 with the
    // reference's pi = 4 atan(1) (src/EllipticSolver2d.cc:44)
    const double pi = 4. * atan(1.0);
    std::vector<double> hx(nx), hy(ny);
    std::vector<float> fx(nx), fy(ny);
    for (int i = 0; i < nx; ++i) { hx[i] = cos((pi * i) / nx); fx[i] = (float)hx[i]; }
    for (int j = 0; j < ny; ++j) { hy[j] = cos((pi * j) / ny); fy[j] = (float)hy[j]; }
    if (cudaMalloc(&x64, sizeof(double) * nx) || cudaMalloc(&y64, sizeof(double) * ny) ||
        cudaMalloc(&x32, sizeof(float) * nx) || cudaMalloc(&y32, sizeof(float) * ny))
        return IBG_ERR_CUDA;
    cudaMemcpy(x64, hx.data(), sizeof(double) * nx, cudaMemcpyHostToDevice);
    cudaMemcpy(y64, hy.data(), sizeof(double) * ny, cudaMemcpyHostToDevice);
    cudaMemcpy(x32, fx.data(), sizeof(float) * nx, cudaMemcpyHostToDevice);
    cudaMemcpy(y32, fy.data(), sizeof(float) * ny, cudaMemcpyHostToDevice);
    return IBG_OK;
}

void CosTables::release() {
    cudaFree(x64); cudaFree(y64); cudaFree(x32); cudaFree(y32);
    x64 = y64 = nullptr;
    x32 = y32 = nullptr;
}

template struct EllipticPlan<double>;
template struct EllipticPlan<float>;

}  // namespace ibg
