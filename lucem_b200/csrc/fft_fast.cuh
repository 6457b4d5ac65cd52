// fft_fast.cuh -- register-resident two-step FFT for power-of-two lengths.
//
// A length N = N1 * N2 transform (N2 >= N1, both powers of two, N2 <= 32) is
// done by N1 threads per sequence, each holding N2 complex values:
//   step 1  thread t holds x[t + N1 i], i < N2, and runs an N2-point DFT in
//           registers, then multiplies by W_N^{t k2};
//   exchange through shared memory (one write, one read);
//   step 2  thread t takes k2 = t + N1 s (s < N2 / N1) and runs N1-point DFTs
//           over n1, giving X[k2 + N2 k1].
// The inverse runs the same steps backwards.  Input and output are in natural
// order; a pointwise product between a forward and an inverse transform (the
// transfer function) needs no exchange at all.  Two exchanges per forward +
// inverse pair, against one per radix stage for a shared-memory FFT.
//
// Register DFTs are in place (radix-2 decimation in frequency forward,
// decimation in time inverse; the bit-reversed order between them is folded
// into compile-time indices) and use twiddle constants computed at compile time: cos/sin of
// 2 pi m / L by exact octant reduction on the integer m and a Taylor
// polynomial on [0, pi/4] (double precision, rounded once to float).  The
// run-time twiddles W_N^{t k2} come from a table the host computes in double
// precision, rearranged per CTA into conflict-free shared tables.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

namespace lucem {
namespace fftc {

constexpr double kHalfPi = 1.57079632679489661923132169163975144;

constexpr double sin_poly(double x) {  // |x| <= pi/4
    double x2 = x * x, term = x, sum = x;
    for (int k = 1; k <= 12; ++k) {
        term *= -x2 / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}

constexpr double cos_poly(double x) {  // |x| <= pi/4
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k <= 12; ++k) {
        term *= -x2 / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}

// cos / sin of 2 pi m / L.
constexpr double cos2pi(long m, long L) {
    m %= L;
    if (m < 0) m += L;
    long q = (4 * m) / L, r = 4 * m - q * L;  // angle = pi/2 (q + r / L)
    double cp = 0, sp = 0;
    if (2 * r <= L) {
        double phi = kHalfPi * (double)r / (double)L;
        cp = cos_poly(phi);
        sp = sin_poly(phi);
    } else {
        double phi = kHalfPi * (double)(L - r) / (double)L;
        cp = sin_poly(phi);
        sp = cos_poly(phi);
    }
    return q == 0 ? cp : (q == 1 ? -sp : (q == 2 ? -cp : sp));
}
constexpr double sin2pi(long m, long L) {
    m %= L;
    if (m < 0) m += L;
    long q = (4 * m) / L, r = 4 * m - q * L;
    double cp = 0, sp = 0;
    if (2 * r <= L) {
        double phi = kHalfPi * (double)r / (double)L;
        cp = cos_poly(phi);
        sp = sin_poly(phi);
    } else {
        double phi = kHalfPi * (double)(L - r) / (double)L;
        cp = sin_poly(phi);
        sp = cos_poly(phi);
    }
    return q == 0 ? sp : (q == 1 ? cp : (q == 2 ? -sp : -cp));
}

// Complex add and subtract as one packed f32x2 instruction each (sm_100
// add.f32x2 / sub.f32x2; the same IEEE result per component as two scalar
// operations).  The subtraction is written in PTX (no CUDA intrinsic for it),
// so it needs no negated copy of its operand.
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) {
    float2 r;
    asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n sub.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 mul(float2 a, float2 w) {
    return make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// a * W_L^K (forward: e^{-2 pi i K / L}; inverse: conjugate).
template <int L, int K, bool INV>
__device__ __forceinline__ float2 rot(float2 a) {
    constexpr int k = ((K % L) + L) % L;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (4 * k == L) {  // -i (forward) / +i (inverse)
        return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    } else if constexpr (2 * k == L) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * k == 3 * L) {  // +i (forward) / -i (inverse)
        return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
    } else {
        constexpr float wr = (float)cos2pi(k, L);
        constexpr float wi = INV ? (float)sin2pi(k, L) : -(float)sin2pi(k, L);
        return make_float2(fmaf(a.x, wr, -a.y * wi), fmaf(a.x, wi, a.y * wr));
    }
}

constexpr int bitrev(int p, int L) {
    int r = 0;
    for (int b = 1; b < L; b <<= 1) {
        r = (r << 1) | (p & 1);
        p >>= 1;
    }
    return r;
}

// One radix-2 butterfly pair of an in-place stage, block b, offset J, half span H.
template <int H, bool INV, bool DIF, int I>
__device__ __forceinline__ void pair(float2 *v) {
    constexpr int b = I / H, j = I % H;
    constexpr int lo = b * 2 * H + j, hi = lo + H;
    float2 a = v[lo], c = v[hi];
    if constexpr (DIF) {
        v[lo] = add(a, c);
        v[hi] = rot<2 * H, j, INV>(sub(a, c));
    } else {
        c = rot<2 * H, j, INV>(c);
        v[lo] = add(a, c);
        v[hi] = sub(a, c);
    }
}

template <int H, bool INV, bool DIF, int... I>
__device__ __forceinline__ void stage(float2 *v, std::integer_sequence<int, I...>) {
    (pair<H, INV, DIF, I>(v), ...);
}

// In-register DFT of length L (power of two), in place.
//   forward (INV = false): decimation in frequency, natural order in,
//     bit-reversed order out (v[p] = X[bitrev(p)]);
//   inverse (INV = true): decimation in time, bit-reversed order in,
//     natural order out (unnormalised).
template <int L, bool INV, int H = (INV ? 1 : L / 2)>
__device__ __forceinline__ void rdft(float2 *v) {
    if constexpr (L >= 2) {
        stage<H, INV, !INV>(v, std::make_integer_sequence<int, L / 2>{});
        if constexpr (!INV && H > 1) rdft<L, INV, H / 2>(v);
        if constexpr (INV && 2 * H < L) rdft<L, INV, 2 * H>(v);
    }
}

// First decimation-in-frequency stage when the upper half of the input is
// zero: (a, 0) -> (a, W_L^j a).
template <int L, int... J>
__device__ __forceinline__ void first_stage_zero_hi(float2 *v, std::integer_sequence<int, J...>) {
    ((v[J + L / 2] = rot<L, J, false>(v[J])), ...);
}

// Decimation-in-time inverse of length L computing only the lower half of
// the output: every stage but the last as rdft, the last one (half span
// L/2, a single block) producing v[j] = v[j] + W^j v[j + L/2] only.
template <int L, int... J>
__device__ __forceinline__ void last_stage_lo(float2 *v, std::integer_sequence<int, J...>) {
    ((v[J] = add(v[J], rot<L, J, true>(v[J + L / 2]))), ...);
}
template <int L, int H = 1>
__device__ __forceinline__ void rdft_inv_lo(float2 *v) {
    if constexpr (2 * H < L) {
        stage<H, true, false>(v, std::make_integer_sequence<int, L / 2>{});
        rdft_inv_lo<L, 2 * H>(v);
    } else {
        last_stage_lo<L>(v, std::make_integer_sequence<int, L / 2>{});
    }
}

// Exchange-buffer layouts.  ColLayout: C sequences per CTA along columns
// (lanes run along c); [N2][N1 * C + PAD] with PAD = C mod 16 so that a half
// warp touches 32 distinct banks.  RowLayout: R sequences per CTA along rows
// (lanes run along t); [R][N2][N1 + 1] (odd pitch), rows padded so that two
// rows in one half warp land 16 banks apart.
template <int N1, int N2, int C>
struct ColLayout {
    static constexpr int P = N1 * C + (C % 16);
    static constexpr int kBuf = N2 * P;
    __device__ __forceinline__ static int idx(int k2, int n1, int c) { return k2 * P + n1 * C + c; }
};
template <int N1, int N2, int R>
struct RowLayout {
    static constexpr int Q = N1 + 1;
    static constexpr int RP0 = N2 * Q;
    static constexpr int RP = N1 >= 16 ? RP0 : RP0 + ((8 - RP0 % 16) + 16) % 16;
    static constexpr int kBuf = R * RP;
    __device__ __forceinline__ static int idx(int k2, int n1, int r) { return r * RP + k2 * Q + n1; }
};

// Two-step transform; thread (c, t), t < N1, c = the sequence in the CTA.
// Run-time twiddles come from two shared tables built once per CTA (see
// build_tables), laid out so that lanes read consecutive entries whichever
// of t or c varies across the warp:
//   tf[k2 * N1 + t]  = W_N^{t k2}   (forward, step 1)
//   ti[n1 * N2 + k2] = W_N^{-n1 k2} (inverse, before the exchange)
template <int N1_, int N2_, class Layout>
struct TwoStep {
    static constexpr int N1 = N1_, N2 = N2_, N = N1 * N2, S = N2 / N1;
    static constexpr int kTables = 2 * N;  // complex entries of tf + ti
    static_assert(N2 % N1 == 0, "N2 must be a multiple of N1");

    // `w` holds W_N^m at w[m * ws], m < N.  Caller synchronises afterwards.
    __device__ __forceinline__ static void build_tables(float2 *tf, float2 *ti, const float2 *w, int ws) {
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            const int k2 = i / N1, t = i % N1;
            tf[i] = w[t * k2 * ws];
            const int n1 = i / N2, kk = i % N2;
            ti[i] = conjf2(w[n1 * kk * ws]);
        }
    }

    // v[i] = x[t + N1 i]  ->  v[s N1 + p] = X[(t + N1 s) + N2 bitrev_N1(p)]
    // (see freq).  Ends synchronised.  ZERO_HI: the input rows N/2 .. N-1
    // are zero (v[i] = 0 for i >= N2/2; zero padding to at least twice the
    // data), so the first butterfly stage reduces to v[i + N2/2] = W v[i].
    template <bool ZERO_HI = false>
    __device__ __forceinline__ static void forward(float2 *v, int t, int c, float2 *xb, const float2 *tf) {
        if constexpr (ZERO_HI && N2 >= 4) {
            first_stage_zero_hi<N2>(v, std::make_integer_sequence<int, N2 / 2>{});
            rdft<N2, false, N2 / 4>(v);
        } else {
            rdft<N2, false>(v);  // v[p] = Y[bitrev(p)]
        }
#pragma unroll
        for (int p = 0; p < N2; ++p) {
            const int k2 = bitrev(p, N2);
            float2 y = k2 ? mul(v[p], tf[k2 * N1 + t]) : v[p];
            xb[Layout::idx(k2, t, c)] = y;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k2 = t + N1 * s;
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) v[s * N1 + n1] = xb[Layout::idx(k2, n1, c)];
            rdft<N1, false>(v + s * N1);
        }
        __syncthreads();
    }

    // Inverse (unnormalised) of the forward layout: v[i] = N x[t + N1 i] on return.
    // LO_ONLY: only the rows 0 .. N/2-1 are wanted (v[i], i < N2/2); the
    // last butterfly stage skips the upper halves, which are left undefined.
    template <bool LO_ONLY = false>
    __device__ __forceinline__ static void inverse(float2 *v, int t, int c, float2 *xb, const float2 *ti) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k2 = t + N1 * s;
            rdft<N1, true>(v + s * N1);  // natural n1
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                float2 z = v[s * N1 + n1];
                if (n1) z = mul(z, ti[n1 * N2 + k2]);
                xb[Layout::idx(k2, n1, c)] = z;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) v[bitrev(k2, N2)] = xb[Layout::idx(k2, t, c)];
        if constexpr (LO_ONLY && N2 >= 4) rdft_inv_lo<N2>(v);
        else rdft<N2, true>(v);
        __syncthreads();
    }

    // Frequency held in value slot j of thread t (forward output layout).
    __host__ __device__ __forceinline__ static constexpr int freq(int t, int j) {
        return (t + N1 * (j / N1)) + N2 * bitrev(j % N1, N1);
    }

    // The slot holding frequency N - freq(t, j) in thread N1 - t, the same
    // for every t >= 1 (mirror pairs of a real transform's packing).
    static constexpr int mirror_slot(int j) {
        const int target = N - freq(1, j);
        for (int q = 0; q < N2; ++q)
            if (freq(N1 - 1, q) == target) return q;
        return -1;
    }
    // Thread 0: the slot holding frequency (N - freq(0, j)) mod N in thread 0
    // itself (j = 0: frequency 0, its own slot).
    static constexpr int mirror_slot0(int j) {
        const int target = (N - freq(0, j)) % N;
        for (int q = 0; q < N2; ++q)
            if (freq(0, q) == target) return q;
        return -1;
    }
};

}  // namespace fftc
}  // namespace lucem
