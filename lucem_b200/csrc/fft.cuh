// fft.cuh -- shared-memory self-sorting (Stockham) FFT for any length whose
// factors are 2, 3, 5 and 7: the generic path of the Richardson-Lucy passes
// (power-of-two lengths take the register-resident transform in
// fft_fast.cuh).
//
// A CTA transforms C independent sequences ("columns") of length n that sit
// in shared memory as buf[row * CP + c] (CP = C + 1: both the column-major
// butterfly accesses and the row-major transposing loads are free of bank
// conflicts).  Lanes run along c.  Each stage reads one buffer and writes the
// other; each thread holds one radix-R butterfly at a time.  Twiddles
// W_n^m = e^{-2 pi i m / n} come from a table computed in double precision on
// the host and rounded once to float (no device sin/cos).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace lucem {
namespace fft {

struct Tw {
    const float2 *t;  // table of length n_table: e^{-2 pi i m / n_table}
    int stride;       // W_n^m = t[m * stride]  (n * stride == n_table)
    __device__ __forceinline__ float2 get(int m, bool inv) const {
        float2 w = t[m * stride];
        if (inv) w.y = -w.y;
        return w;
    }
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// Add as one packed f32x2 instruction (sm_100), same result as two scalar adds.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 mul_mi(float2 a, bool inv) {
    return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
struct Dft;

template <>
struct Dft<2> {
    __device__ __forceinline__ static void run(float2 *v, bool) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <>
struct Dft<4> {
    __device__ __forceinline__ static void run(float2 *v, bool inv) {
        float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        float2 s13 = cadd(v[1], v[3]), d13 = mul_mi(csub(v[1], v[3]), inv);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    }
};

template <>
struct Dft<8> {
    __device__ __forceinline__ static void run(float2 *v, bool inv) {
        // Two 4-point DFTs over even / odd inputs, then W_8^k on the odd half.
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e, inv);
        Dft<4>::run(o, inv);
        const float h = 0.70710678118654752440f;  // sqrt(2)/2
        // W_8^1 = (h, -h), W_8^2 = -i, W_8^3 = (-h, -h)  (forward)
        float2 o1 = inv ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                        : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
        float2 o2 = mul_mi(o[2], inv);
        float2 o3 = inv ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                        : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

// cos / sin(2 pi m / R), m = 1 .. (R-1)/2, for the odd radices.
template <int R> struct OddConst;
template <> struct OddConst<3> {
    __device__ static constexpr float c(int) { return -5.000000000e-01f; }
    __device__ static constexpr float s(int) { return 8.660254038e-01f; }
};
template <> struct OddConst<5> {
    __device__ static constexpr float c(int m) { return m == 1 ? 3.090169944e-01f : -8.090169944e-01f; }
    __device__ static constexpr float s(int m) { return m == 1 ? 9.510565163e-01f : 5.877852523e-01f; }
};
template <> struct OddConst<7> {
    __device__ static constexpr float c(int m) {
        return m == 1 ? 6.234898019e-01f : (m == 2 ? -2.225209340e-01f : -9.009688679e-01f);
    }
    __device__ static constexpr float s(int m) {
        return m == 1 ? 7.818314825e-01f : (m == 2 ? 9.749279122e-01f : 4.338837391e-01f);
    }
};

// Odd radix R = 2h+1: pair the inputs r and R-r, X[k] and X[R-k] share the
// cosine sums and differ in the sign of the sine sums.
template <int R>
struct DftOdd {
    __device__ __forceinline__ static void run(float2 *v, bool inv) {
        constexpr int H = (R - 1) / 2;
        float2 sp[H], sm[H];
        float2 x0 = v[0];
#pragma unroll
        for (int r = 1; r <= H; ++r) {
            sp[r - 1] = cadd(v[r], v[R - r]);
            sm[r - 1] = csub(v[r], v[R - r]);
        }
        float2 sum = x0;
#pragma unroll
        for (int r = 0; r < H; ++r) sum = cadd(sum, sp[r]);
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            float2 a = x0, b = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 1; r <= H; ++r) {
                const int m = (k * r) % R;
                const float c = OddConst<R>::c(m <= H ? m : R - m);
                const float s = m <= H ? OddConst<R>::s(m) : -OddConst<R>::s(R - m);
                a.x = fmaf(c, sp[r - 1].x, a.x);
                a.y = fmaf(c, sp[r - 1].y, a.y);
                b.x = fmaf(s, sm[r - 1].x, b.x);
                b.y = fmaf(s, sm[r - 1].y, b.y);
            }
            // forward: X[k] = a - i b, X[R-k] = a + i b
            float2 ib = make_float2(-b.y, b.x);
            v[k] = inv ? cadd(a, ib) : csub(a, ib);
            v[R - k] = inv ? csub(a, ib) : cadd(a, ib);
        }
        v[0] = sum;
    }
};
template <> struct Dft<3> : DftOdd<3> {};
template <> struct Dft<5> : DftOdd<5> {};
template <> struct Dft<7> : DftOdd<7> {};

// ---- self-sorting (Stockham) transform, two buffers ----------------------
// Natural order in and out.  Stage with radix R after Ns = product of the
// earlier radices, butterfly j in [0, n/R), k = j mod Ns:
//   v[r] = src[j + r n/R] * W_{Ns R}^{k r};  v = DFT_R(v);
//   dst[(j / Ns) Ns R + k + r Ns] = v[r].
template <int R>
__device__ __forceinline__ void stockham_stage(const float2 *src, float2 *dst, int n, int C, int CP, int Ns,
                                               const Tw &tw, bool inv) {
    const int nR = n / R;
    const int nb = nR * C;
    const int tws = n / (Ns * R);
    for (int item = threadIdx.x; item < nb; item += blockDim.x) {
        const int c = item % C, j = item / C;
        const int k = j % Ns;
        float2 v[R];
        v[0] = src[j * CP + c];
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 x = src[(j + r * nR) * CP + c];
            v[r] = k ? cmul(x, tw.get(k * r * tws, inv)) : x;
        }
        Dft<R>::run(v, inv);
        float2 *d = dst + ((j / Ns) * Ns * R + k) * CP + c;
#pragma unroll
        for (int r = 0; r < R; ++r) d[r * Ns * CP] = v[r];
    }
    __syncthreads();
}

// Returns the buffer (a or b) that holds the result.  The caller synchronises
// after filling a.
__device__ __forceinline__ float2 *stockham(float2 *a, float2 *b, int n, int C, int CP, const int *radix,
                                            int nstages, const Tw &tw, bool inv) {
    int Ns = 1;
    for (int i = 0; i < nstages; ++i) {
        const int R = radix[i];
        switch (R) {
        case 8: stockham_stage<8>(a, b, n, C, CP, Ns, tw, inv); break;
        case 4: stockham_stage<4>(a, b, n, C, CP, Ns, tw, inv); break;
        case 2: stockham_stage<2>(a, b, n, C, CP, Ns, tw, inv); break;
        case 3: stockham_stage<3>(a, b, n, C, CP, Ns, tw, inv); break;
        case 5: stockham_stage<5>(a, b, n, C, CP, Ns, tw, inv); break;
        case 7: stockham_stage<7>(a, b, n, C, CP, Ns, tw, inv); break;
        default: break;
        }
        Ns *= R;
        float2 *t = a;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace fft
}  // namespace lucem
