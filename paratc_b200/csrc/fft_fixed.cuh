// fft_fixed.cuh -- batched complex FFTs whose length is a compile-time
// constant, for the transforms of the pressure Poisson solve.
//
// A CTA transforms B sequences of length N held in shared memory as
// buf[e*PITCH + b] (element e of sequence b; b fastest, so that a warp's 32
// lanes touch consecutive 16-byte words).  The transform is a sequence of
// Stockham autosort passes with radices 16, 8, 4, 2, 3 and 5: every index,
// stride and loop bound is a constant, so a pass is loads, constant-twiddle
// butterflies and stores, with no integer division at run time.  Pass s of
// radix R after passes whose radices multiply to NS reads element j + r*N/R
// (r < R) of butterfly j, multiplies by exp(-+2 pi i (j mod NS) r / (NS R))
// and writes element (j - j mod NS) R + j mod NS + r NS: the classic Stockham
// formulation, done in place (all threads load their inputs to registers, the
// block synchronises, then all store).  Inter-pass twiddles come from a table
// tw[m] = exp(-2 pi i m / N) that the caller stages in shared memory.
#pragma once
#include "common.cuh"

namespace ptc {
namespace ff {

// radix schedule of N = 2^a 3^b 5^c: the power of two in ceil(a/maxbits)
// passes of radix <= 2^maxbits as even as possible, then radix-3 and radix-5
// passes
struct Sched {
    int np;
    int r[12];
};

__host__ __device__ constexpr Sched make_sched(int n, int maxbits = 4) {
    Sched s{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    int a = 0;
    while (n % 2 == 0) { n /= 2; a++; }
    const int p2 = (a + maxbits - 1) / maxbits;
    for (int q = 0; q < p2; q++) s.r[s.np++] = 1 << ((a + q) / p2);
    while (n % 3 == 0 && s.np < 12) { n /= 3; s.r[s.np++] = 3; }
    while (n % 5 == 0 && s.np < 12) { n /= 5; s.r[s.np++] = 5; }
    if (n != 1) s.np = -1;
    return s;
}

__host__ __device__ constexpr int sched_rmax(int n) {
    const Sched s = make_sched(n);
    int m = 1;
    for (int q = 0; q < s.np; q++) m = s.r[q] > m ? s.r[q] : m;
    return m;
}

// product of the radices of passes 0..S-1
__host__ __device__ constexpr int sched_ns(int n, int S, int maxbits = 4) {
    const Sched s = make_sched(n, maxbits);
    int p = 1;
    for (int q = 0; q < S; q++) p *= s.r[q];
    return p;
}

// cos and sin of 2 pi k / 16
__host__ __device__ constexpr double c16(int k) {
    switch (k & 15) {
        case 0: return 1.0;
        case 1: return 0.92387953251128675613;
        case 2: return 0.70710678118654752440;
        case 3: return 0.38268343236508977173;
        case 4: return 0.0;
        case 5: return -0.38268343236508977173;
        case 6: return -0.70710678118654752440;
        case 7: return -0.92387953251128675613;
        case 8: return -1.0;
        case 9: return -0.92387953251128675613;
        case 10: return -0.70710678118654752440;
        case 11: return -0.38268343236508977173;
        case 12: return 0.0;
        case 13: return 0.38268343236508977173;
        case 14: return 0.70710678118654752440;
        default: return 0.92387953251128675613;
    }
}
__host__ __device__ constexpr double s16(int k) { return c16(k - 4); }

// v * exp(DIR 2 pi i k / M) for M in {2, 4, 8, 16}, with the trivial angles
// done exactly
// (C: double2, or float2 for the FP32 arithmetic of the FP32 storage form;
// the constants are rounded to C's real type)
template <int M, int K, int DIR, class C>
__device__ __forceinline__ C rot(C v) {
    using R = typename Cx<C>::R;
    constexpr int k16 = (K * (16 / M)) & 15;
    if constexpr (k16 == 0) return v;
    else if constexpr (k16 == 8) return Cx<C>::make(-v.x, -v.y);
    else if constexpr (k16 == 4) return DIR < 0 ? Cx<C>::make(v.y, -v.x) : Cx<C>::make(-v.y, v.x);
    else if constexpr (k16 == 12) return DIR < 0 ? Cx<C>::make(-v.y, v.x) : Cx<C>::make(v.y, -v.x);
    else {
        constexpr R c = (R)c16(k16), s = (R)(DIR * s16(k16));
        return Cx<C>::make(v.x * c - v.y * s, v.x * s + v.y * c);
    }
}

template <int DIR, class C>
__device__ __forceinline__ void dft2(C* v) {
    const C t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}

template <int DIR, class C>
__device__ __forceinline__ void dft3(C* v) {
    using R = typename Cx<C>::R;
    const R c = (R)-0.5, s = (R)(DIR * 0.86602540378443864676);  // cos, sin of 2 pi / 3
    const C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const C mm = Cx<C>::make(v[0].x + c * t1.x, v[0].y + c * t1.y);
    const C it = Cx<C>::make(-s * t2.y, s * t2.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(mm, it);
    v[2] = csub(mm, it);
}

template <int DIR, class C>
__device__ __forceinline__ void dft5(C* v) {
    using R = typename Cx<C>::R;
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;  // cos 2pi/5, cos 4pi/5
    const R s1 = (R)(DIR * 0.95105651629515357212), s2 = (R)(DIR * 0.58778525229247312917);
    const C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const C m1 = Cx<C>::make(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const C m2 = Cx<C>::make(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const C n1 = Cx<C>::make(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
    const C n2 = Cx<C>::make(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
    const C in1 = Cx<C>::make(-n1.y, n1.x), in2 = Cx<C>::make(-n2.y, n2.x);
    v[0] = Cx<C>::make(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
    v[1] = cadd(m1, in1);
    v[4] = csub(m1, in1);
    v[2] = cadd(m2, in2);
    v[3] = csub(m2, in2);
}

// radix-2 combination of the half-length DFTs of the even (E) and odd (O)
// samples: X[k] = E[k] + W^k O[k], X[k + H] = E[k] - W^k O[k], W = exp(DIR 2 pi i / 2H)
template <int H, int DIR, int K = 0, class C>
__device__ __forceinline__ void combine(const C* E, const C* O, C* X) {
    if constexpr (K < H) {
        const C t = rot<2 * H, K, DIR>(O[K]);
        X[K] = cadd(E[K], t);
        X[K + H] = csub(E[K], t);
        combine<H, DIR, K + 1>(E, O, X);
    }
}

template <int R, int DIR, class C>
__device__ __forceinline__ void dft(C* v) {
    if constexpr (R == 2) dft2<DIR>(v);
    else if constexpr (R == 3) dft3<DIR>(v);
    else if constexpr (R == 5) dft5<DIR>(v);
    else {
        constexpr int H = R / 2;
        C e[H], o[H];
#pragma unroll
        for (int q = 0; q < H; q++) { e[q] = v[2 * q]; o[q] = v[2 * q + 1]; }
        dft<H, DIR>(e);
        dft<H, DIR>(o);
        combine<H, DIR>(e, o, v);
    }
}

// barrier of the P threads that run the transform: the whole CTA (BAR = 0)
// or named barrier BAR over the first P threads (warp-specialised kernels)
template <int BAR, int P>
__device__ __forceinline__ void group_sync() {
    if constexpr (BAR == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;\n" ::"n"(BAR), "n"(P) : "memory");
}

// barrier of the same group that also returns, to every thread, whether any
// thread of the group passed a true predicate (a uniform decision)
template <int BAR, int P>
__device__ __forceinline__ bool group_any(bool pred) {
    if constexpr (BAR == 0) {
        return __syncthreads_or(pred ? 1 : 0) != 0;
    } else {
        unsigned r;
        asm volatile(
            "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
            : "=r"(r)
            : "r"(pred ? 1u : 0u), "n"(BAR), "n"(P)
            : "memory");
        return r != 0;
    }
}

// One Stockham pass of radix R (passes before it multiply to NS) over B
// sequences of length N, P threads.  LD(e, b) loads element e of sequence b,
// ST(e, b, v) stores it; SYNC_MID puts a block barrier between all loads and
// all stores (an in-place pass on shared memory).  tw: exp(-2 pi i m / N).
template <int N, int B, int P, int R, int NS, int DIR, bool SYNC_MID, class LD, class ST, int BAR = 0,
          class C = double2>
__device__ __forceinline__ void pass(const LD& ld, const ST& st, const C* tw, int tid) {
    constexpr int NB = N / R;
    constexpr int TOT = B * NB;
    constexpr int PER = (TOT + P - 1) / P;
    constexpr int TS = N / (NS * R);
    C v[PER][R];
    int jb[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
        const int t = tid + u * P;
        jb[u] = -1;
        if (TOT % P == 0 || t < TOT) {
            const int b = t % B, j = t / B;
            const int kk = j % NS;
#pragma unroll
            for (int r = 0; r < R; r++) v[u][r] = ld(j + r * NB, b);
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    const C w = tw[kk * r * TS];
                    v[u][r] = (DIR < 0) ? cmul(v[u][r], w) : cmulc(v[u][r], w);
                }
            }
            dft<R, DIR>(v[u]);
            jb[u] = ((j - kk) * R + kk) * B + b;  // output element * B + b
        }
    }
    if constexpr (SYNC_MID) group_sync<BAR, P>();
#pragma unroll
    for (int u = 0; u < PER; u++) {
        if (TOT % P == 0 || jb[u] >= 0) {
            const int b = jb[u] % B, e0 = jb[u] / B;
#pragma unroll
            for (int r = 0; r < R; r++) st(e0 + r * NS, b, v[u][r]);
        }
    }
}

// shared-memory accessors of the layout buf[e*PITCH + b]
template <int PITCH, class C = double2>
struct SmemLd {
    const C* buf;
    __device__ __forceinline__ C operator()(int e, int b) const { return buf[e * PITCH + b]; }
};
template <int PITCH, class C = double2>
struct SmemSt {
    C* buf;
    __device__ __forceinline__ void operator()(int e, int b, C v) const { buf[e * PITCH + b] = v; }
};

// shared-memory accessors with the sequence index major: element e of
// sequence b at buf[b*PITCH + e], or at buf[b*PITCH + swz8(e)] with SWZ:
// swz8(e) = e ^ ((e >> 3) & 7) permutes each aligned group of eight 16-byte
// words, so that the stores of a first Stockham pass (element j*R + r for
// the lanes' consecutive j, all in one bank group when R is 8 or 16) and the
// loads of the next one both spread over the eight bank groups
__device__ __forceinline__ int swz8(int e) { return e ^ ((e >> 3) & 7); }
template <int PITCH, bool SWZ = false, class C = double2>
struct SmemLdT {
    const C* buf;
    __device__ __forceinline__ C operator()(int e, int b) const { return buf[b * PITCH + (SWZ ? swz8(e) : e)]; }
};
template <int PITCH, bool SWZ = false, class C = double2>
struct SmemStT {
    C* buf;
    __device__ __forceinline__ void operator()(int e, int b, C v) const { buf[b * PITCH + (SWZ ? swz8(e) : e)] = v; }
};

// passes S..END-1 in place on shared memory, each followed by a barrier;
// TRANSPOSED selects the layout buf[b*PITCH + e] instead of buf[e*PITCH + b];
// BAR != 0 synchronises only the P transforming threads (named barrier BAR);
// SWZ (TRANSPOSED, N a multiple of 8) keeps the values between passes in the
// swizzled order: pass 0 reads plain and writes swizzled, the last pass
// reads swizzled and writes plain
template <int N, int B, int PITCH, int P, int DIR, int S, int END, int MAXBITS = 4, bool TRANSPOSED = false,
          int BAR = 0, bool SWZ = false, class C = double2>
__device__ __forceinline__ void smem_passes(C* buf, const C* tw, int tid) {
    constexpr Sched SC = make_sched(N, MAXBITS);
    static_assert(!SWZ || (TRANSPOSED && N % 8 == 0), "the swizzle permutes whole groups of eight");
    if constexpr (S < END) {
        constexpr int R = SC.r[S];
        constexpr int NS = sched_ns(N, S, MAXBITS);
        constexpr bool SIN = SWZ && S > 0, SOUT = SWZ && S + 1 < END;
        if constexpr (TRANSPOSED)
            pass<N, B, P, R, NS, DIR, true, SmemLdT<PITCH, SIN, C>, SmemStT<PITCH, SOUT, C>, BAR>(
                SmemLdT<PITCH, SIN, C>{buf}, SmemStT<PITCH, SOUT, C>{buf}, tw, tid);
        else
            pass<N, B, P, R, NS, DIR, true, SmemLd<PITCH, C>, SmemSt<PITCH, C>, BAR>(SmemLd<PITCH, C>{buf},
                                                                                   SmemSt<PITCH, C>{buf}, tw, tid);
        group_sync<BAR, P>();
        smem_passes<N, B, PITCH, P, DIR, S + 1, END, MAXBITS, TRANSPOSED, BAR, SWZ, C>(buf, tw, tid);
    }
}

// launch shape of a length-N transform: B sequences per CTA, P threads (one
// butterfly of the largest radix per thread)
template <int N>
struct Shape {
    static constexpr int RMAX = sched_rmax(N);
    static constexpr int PMAX = N <= 256 ? 128 : 256;
    static constexpr int bcalc() {
        int b = 64;
        while (b > 1 && b * N / RMAX > PMAX) b /= 2;
        return b;
    }
    static constexpr int B = bcalc();
    static constexpr int P = B * N / RMAX;
};

}  // namespace ff
}  // namespace ptc
