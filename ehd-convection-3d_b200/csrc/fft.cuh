// fft.cuh -- small complex DFTs in registers and Stockham passes with
// compile-time radix, for the x and y transforms of the Poisson solve.
//
// Conventions: sign S = -1 is the forward transform exp(-2 pi i jk/N), S = +1
// the inverse, both unnormalised.  `tw` points to the table
// tw[m] = exp(-2 pi i m / N) of the whole transform (in shared memory); a DFT
// of size P inside it reads W_P^m = tw[m * step] with step = N / P.
#pragma once

#include "common.cuh"

namespace ehd {
namespace fft {

template <typename R2> __device__ __forceinline__ R2 add(R2 a, R2 b) { return {a.x + b.x, a.y + b.y}; }
template <typename R2> __device__ __forceinline__ R2 sub(R2 a, R2 b) { return {a.x - b.x, a.y - b.y}; }
template <typename R2> __device__ __forceinline__ R2 mul(R2 a, R2 b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R2, typename R> __device__ __forceinline__ R2 scale(R2 a, R s) { return {a.x * s, a.y * s}; }
// i * S * a
template <int S, typename R2> __device__ __forceinline__ R2 rot(R2 a) {
    return S > 0 ? R2{-a.y, a.x} : R2{a.y, -a.x};
}
// a * W for the forward table entry W, conjugated for the inverse
template <int S, typename R2> __device__ __forceinline__ R2 twmul(R2 a, R2 w) {
    if (S > 0) w.y = -w.y;
    return mul(a, w);
}

template <int P, int S, typename R2> struct Dft;

template <int S, typename R2> struct Dft<1, S, R2> {
    __device__ __forceinline__ static void run(R2 *, const R2 *, int) {}
};
template <int S, typename R2> struct Dft<2, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *, int) {
        const R2 a = v[0];
        v[0] = add(a, v[1]);
        v[1] = sub(a, v[1]);
    }
};
template <int S, typename R2> struct Dft<3, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *, int) {
        using R = decltype(v[0].x);
        const R h3 = (R)0.86602540378443864676;  // sqrt(3)/2
        const R2 t1 = add(v[1], v[2]);
        const R2 t2 = sub(v[0], scale(t1, (R)0.5));
        const R2 t3 = rot<S>(scale(sub(v[1], v[2]), h3));
        v[0] = add(v[0], t1);
        v[1] = add(t2, t3);
        v[2] = sub(t2, t3);
    }
};
template <int S, typename R2> struct Dft<4, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *, int) {
        const R2 s02 = add(v[0], v[2]), d02 = sub(v[0], v[2]);
        const R2 s13 = add(v[1], v[3]), d13 = rot<S>(sub(v[1], v[3]));
        v[0] = add(s02, s13);
        v[1] = add(d02, d13);
        v[2] = sub(s02, s13);
        v[3] = sub(d02, d13);
    }
};
template <int S, typename R2> struct Dft<5, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *, int) {
        using R = decltype(v[0].x);
        const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
        const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
        const R2 t1 = add(v[1], v[4]), t2 = add(v[2], v[3]);
        const R2 t3 = sub(v[1], v[4]), t4 = sub(v[2], v[3]);
        const R2 a1 = add(v[0], add(scale(t1, c1), scale(t2, c2)));
        const R2 a2 = add(v[0], add(scale(t1, c2), scale(t2, c1)));
        const R2 b1 = rot<S>(add(scale(t3, s1), scale(t4, s2)));
        const R2 b2 = rot<S>(sub(scale(t3, s2), scale(t4, s1)));
        v[0] = add(v[0], add(t1, t2));
        v[1] = add(a1, b1);
        v[4] = sub(a1, b1);
        v[2] = add(a2, b2);
        v[3] = sub(a2, b2);
    }
};

// Composite size A*B (Cooley-Tukey, natural order in and out): DFT_A on the
// stride-B subsequences, twiddle W_AB^(n2 k1), DFT_B on the contiguous blocks.
template <int A, int B, int S, typename R2>
__device__ __forceinline__ void dft_ab(R2 *v, const R2 *tw, int step) {
    R2 t[A];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = v[n2 + B * n1];
        Dft<A, S, R2>::run(t, tw, step * B);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) v[n2 + B * k1] = t[k1];
    }
#pragma unroll
    for (int n2 = 1; n2 < B; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < A; ++k1)
            v[n2 + B * k1] = twmul<S>(v[n2 + B * k1], tw[n2 * k1 * step]);
    R2 out[A * B];
    R2 u[B];
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) u[n2] = v[n2 + B * k1];
        Dft<B, S, R2>::run(u, tw, step * A);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) out[k1 + A * k2] = u[k2];
    }
#pragma unroll
    for (int i = 0; i < A * B; ++i) v[i] = out[i];
}

template <int S, typename R2> struct Dft<8, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *tw, int step) { dft_ab<2, 4, S>(v, tw, step); }
};
template <int S, typename R2> struct Dft<16, S, R2> {
    __device__ __forceinline__ static void run(R2 *v, const R2 *tw, int step) { dft_ab<4, 4, S>(v, tw, step); }
};

// padded shared-memory index: one spare element per 16 breaks the bank
// conflicts of the strided stores of the first pass
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + (n >> 4); }

// One Stockham pass of radix R over a length-N transform held (padded) in
// `buf`; butterfly j < N/R.  The caller synchronises between the load/compute
// half and the store half (the pass is in place).
template <int N, int R, int NS, int S, typename R2>
__device__ __forceinline__ void pass_compute(const R2 *buf, const R2 *tw, int j, R2 (&v)[R]) {
    const int k = j % NS;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[pad(j + r * (N / R))];
    if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = twmul<S>(v[r], tw[r * k * (N / (NS * R))]);
    }
    Dft<R, S, R2>::run(v, tw, N / R);
}
template <int N, int R, int NS, typename R2>
__device__ __forceinline__ void pass_store(R2 *buf, int j, const R2 (&v)[R]) {
    const int k = j % NS;
    const int base = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[pad(base + r * NS)] = v[r];
}

template <int N, int R, int NS, int S, typename R2>
__device__ __forceinline__ void pass(R2 *buf, const R2 *tw, int j) {
    R2 v[R];
    const bool act = j < N / R;
    if (act) pass_compute<N, R, NS, S>(buf, tw, j, v);
    __syncthreads();
    if (act) pass_store<N, R, NS>(buf, j, v);
    __syncthreads();
}

// Pass schedules of the compile-time sizes; G = threads per transform, a
// divisor of 256 and at least the butterflies of every pass.
template <int N> struct Plan;
template <> struct Plan<64> {
    static constexpr int G = 8;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<64, 8, 1, S>(b, tw, j);
        pass<64, 8, 8, S>(b, tw, j);
    }
};
template <> struct Plan<128> {
    static constexpr int G = 16;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<128, 8, 1, S>(b, tw, j);
        pass<128, 16, 8, S>(b, tw, j);
    }
};
template <> struct Plan<256> {
    static constexpr int G = 16;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<256, 16, 1, S>(b, tw, j);
        pass<256, 16, 16, S>(b, tw, j);
    }
};
// mixed radix (the grids of the T sweeps: 48, 80, 96 nodes, and their odd
// extensions 2 (NZ - 1) = 48, 80, 96)
template <> struct Plan<48> {
    static constexpr int G = 16;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<48, 16, 1, S>(b, tw, j);
        pass<48, 3, 16, S>(b, tw, j);
    }
};
template <> struct Plan<80> {
    static constexpr int G = 16;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<80, 16, 1, S>(b, tw, j);
        pass<80, 5, 16, S>(b, tw, j);
    }
};
template <> struct Plan<96> {
    static constexpr int G = 32;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<96, 8, 1, S>(b, tw, j);
        pass<96, 4, 8, S>(b, tw, j);
        pass<96, 3, 32, S>(b, tw, j);
    }
};
template <> struct Plan<512> {
    static constexpr int G = 64;
    template <int S, typename R2> __device__ static void run(R2 *b, const R2 *tw, int j) {
        pass<512, 8, 1, S>(b, tw, j);
        pass<512, 8, 8, S>(b, tw, j);
        pass<512, 8, 64, S>(b, tw, j);
    }
};

// ---- warp-synchronous transforms ----
// The G <= 32 threads of a transform lie in one warp (t = lane % G) and
// handle the butterflies j = t, t + G, ... of every pass; the warp
// synchronises between a pass's loads and its stores, so every pass may work
// in place.  The first pass takes its inputs from ld(m) and the last hands
// each output m to st(m, value), so a caller gathers, scatters and scales on
// the way in and out; the passes in between go through buf (padded, as
// pass()).  The caller synchronises the warp before it reads what st wrote.
template <int N, int R, int G, int S, typename R2, typename Ld>
__device__ __forceinline__ void wpass_first(R2 *buf, const R2 *tw, int t, Ld ld) {
    constexpr int NB = N / R, BPT = (NB + G - 1) / G;
    R2 v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + G * b;
        if (j < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[b][r] = ld(j + r * NB);
            Dft<R, S, R2>::run(v[b], tw, NB);
        }
    }
    __syncwarp();
#pragma unroll
    for (int b = 0; b < BPT; ++b)
        if (t + G * b < NB) pass_store<N, R, 1>(buf, t + G * b, v[b]);
    __syncwarp();
}
template <int N, int R, int NS, int G, int S, typename R2>
__device__ __forceinline__ void wpass(R2 *buf, const R2 *tw, int t) {
    constexpr int NB = N / R, BPT = (NB + G - 1) / G;
    R2 v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b)
        if (t + G * b < NB) pass_compute<N, R, NS, S>(buf, tw, t + G * b, v[b]);
    __syncwarp();
#pragma unroll
    for (int b = 0; b < BPT; ++b)
        if (t + G * b < NB) pass_store<N, R, NS>(buf, t + G * b, v[b]);
    __syncwarp();
}
template <int N, int R, int NS, int G, int S, typename R2, typename St>
__device__ __forceinline__ void wpass_last(const R2 *buf, const R2 *tw, int t, St st) {
    constexpr int NB = N / R, BPT = (NB + G - 1) / G;
    R2 v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b)
        if (t + G * b < NB) pass_compute<N, R, NS, S>(buf, tw, t + G * b, v[b]);
    __syncwarp();
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + G * b;
        if (j < NB) {
            const int base = (j / NS) * NS * R + j % NS;
#pragma unroll
            for (int r = 0; r < R; ++r) st(base + r * NS, v[b][r]);
        }
    }
}

// A transform of sign S1, a pointwise map mid(k, X[k]) of its output, a
// transform of sign S2, for N = R * R by G = R threads.  The first
// transform's last pass leaves the outputs k = t + R r in the registers that
// the second's first pass reads as its inputs t + R r, so the spectrum never
// goes through buf.
template <int N, int R, int S1, int S2, typename R2, typename Ld, typename Mid, typename St>
__device__ __forceinline__ void wfilter_sq(R2 *buf, const R2 *tw, int t, Ld ld, Mid mid, St st) {
    static_assert(R * R == N, "square sizes only");
    R2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ld(t + R * r);
    __syncwarp();  // ld may read buf
    Dft<R, S1, R2>::run(v, tw, R);
    pass_store<N, R, 1>(buf, t, v);
    __syncwarp();
    pass_compute<N, R, R, S1>(buf, tw, t, v);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = mid(t + R * r, v[r]);
    Dft<R, S2, R2>::run(v, tw, R);
    __syncwarp();
    pass_store<N, R, 1>(buf, t, v);
    __syncwarp();
    pass_compute<N, R, R, S2>(buf, tw, t, v);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) st(t + R * r, v[r]);
}

template <int N> struct WPlan;
template <> struct WPlan<64> {
    static constexpr int G = 8;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<64, 8, G, S>(b, tw, t, ld);
        wpass_last<64, 8, 8, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<128> {
    static constexpr int G = 16;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<128, 8, G, S>(b, tw, t, ld);
        wpass_last<128, 16, 8, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<256> {
    static constexpr int G = 16;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<256, 16, G, S>(b, tw, t, ld);
        wpass_last<256, 16, 16, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<48> {
    static constexpr int G = 16;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<48, 16, G, S>(b, tw, t, ld);
        wpass_last<48, 3, 16, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<80> {
    static constexpr int G = 16;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<80, 16, G, S>(b, tw, t, ld);
        wpass_last<80, 5, 16, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<96> {
    static constexpr int G = 32;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<96, 8, G, S>(b, tw, t, ld);
        wpass<96, 4, 8, G, S>(b, tw, t);
        wpass_last<96, 3, 32, G, S>(b, tw, t, st);
    }
};
template <> struct WPlan<512> {
    static constexpr int G = 32;
    template <int S, typename R2, typename Ld, typename St>
    __device__ static void run(R2 *b, const R2 *tw, int t, Ld ld, St st) {
        wpass_first<512, 8, G, S>(b, tw, t, ld);
        wpass<512, 8, 8, G, S>(b, tw, t);
        wpass_last<512, 8, 64, G, S>(b, tw, t, st);
    }
};

// In-place transform of one row of a tile (padded, length N) by its G
// threads, ending with a block barrier as Plan<N>::run does: warp-synchronous
// where the warp plan has the block plan's G, block-wide otherwise (N = 512).
template <int N, int S, typename R2>
__device__ __forceinline__ void run_tile(R2 *b, const R2 *tw, int j) {
    if constexpr (WPlan<N>::G == Plan<N>::G) {
        WPlan<N>::template run<S>(
            b, tw, j, [&](int m) { return b[pad(m)]; }, [&](int m, R2 v) { b[pad(m)] = v; });
        __syncthreads();
    } else {
        Plan<N>::template run<S>(b, tw, j);
    }
}

}  // namespace fft
}  // namespace ehd
