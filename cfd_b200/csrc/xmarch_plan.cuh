// xmarch_plan.cuh - launch geometry, thread roles and y-step sequence of the x-line pass
// marching in y (k_xmarch, xmarch.cuh).  Pure index arithmetic, callable from host code:
// the kernel computes its roles and steps with these functions, and tests/xmarch_check.cu
// checks them on the CPU (bounds of every shared-memory index, each work item taken once,
// shuffle partners, and that every u-plane and v-plane is produced once from the right
// planes).
#pragma once

#include <cuda_runtime.h>

namespace cfd {

// Row pitches (in 8-byte words for FP32 complex) of the two exchanges: the physical phase
// reads the inverse exchange and writes the forward one with the three lines of a triple
// side by side, so the line pitches put the three roles of a warp 10 and 20 = 4 bank pairs
// apart (inverse) and 2*5 and 4*5 apart (forward, where a lane's lines are 2 apart): each
// bank pair then sees at most two of the 30 lanes, the minimum for 8-byte accesses.
__host__ __device__ constexpr int xmarch_pitch(int x, int r) { return x + (((r - x % 16) % 16) + 16) % 16; }
__host__ __device__ constexpr int xmarch_l1(int n1, int n2) { return xmarch_pitch(n1 * (n2 + 1), 10); }
__host__ __device__ constexpr int xmarch_l2(int n1, int n2) { return xmarch_pitch(n2 * (n1 + 1), 5); }

// threads of a k_xmarch CTA with RW rows (RW/2 row pairs) and the split N1 x N2
__host__ __device__ constexpr int xmarch_threads(int n1, int n2, int rw) {
    const int pairs = rw / 2;
    int nt = 3 * pairs * n2;                          // step 1: 3 lines per pair
    if (6 * pairs * n2 > nt) nt = 6 * pairs * n2;     // step 2': 6 lines per pair
    const int tw = 32 * ((pairs * n1 + 9) / 10);      // triples, 10 per warp
    if (tw > nt) nt = tw;
    return (nt + 31) / 32 * 32;
}

// dynamic shared memory (elements of the complex type): inverse and forward exchanges,
// the per-thread history and the twiddle table
__host__ __device__ constexpr long long xmarch_smem_elems(int n1, int n2, int rw) {
    const int pairs = rw / 2;
    const long long l1 = xmarch_l1(n1, n2), l2 = xmarch_l2(n1, n2);
    return 3LL * pairs * l1 + 6LL * pairs * l2 + (long long)n2 * xmarch_threads(n1, n2, rw) +
           (long long)n1 * (n2 + 1);
}

// The roles of thread t of a CTA with RW rows and the split N1 x N2.
struct XMRoles {
    // step 1: inverse N1-point DFT of line b1 (3 per row pair: A = u_r + i v_r,
    // B = u_r+1 + i v_r+1, C = w_r + i w_r+1), element column n2
    bool act1;
    int b1, n2, p1, role1;
    // physical phase: lane of triple g3 (10 per warp, lanes 30 and 31 idle) with role
    // 0 = A, 1 = B, 2 = C; pair p2, subsequence k1, inverse line b2; the lanes whose u and
    // face value of w the lane reads by shuffle
    bool act2;
    int role, p2, k1, b2, src1, src2;
    // step 2': forward N1-point DFT of forward line bf (clamped to bfc), element kb; the lane
    // holding X_N-k; the line's pair, role and which of the role's two lines
    bool act3;
    int bf, kb, bfc, partner, p3, role3, j3;
};

__host__ __device__ inline XMRoles xmarch_roles(int t, int RW, int N1, int N2) {
    XMRoles r;
    const int pairs = RW >> 1;
    const int NLI = 3 * pairs, NLF = 6 * pairs, NTRI = pairs * N1;
    r.act1 = t < NLI * N2;
    r.b1 = t / N2;
    r.n2 = t - r.b1 * N2;
    r.p1 = r.b1 / 3;
    r.role1 = r.b1 - 3 * r.p1;
    const int lane = t & 31;
    const int g3 = (t >> 5) * 10 + lane / 3;
    r.role = lane - 3 * (lane / 3);
    r.act2 = lane < 30 && g3 < NTRI;
    const int gq = r.act2 ? g3 : 0;
    r.p2 = gq / N1;
    r.k1 = gq - r.p2 * N1;
    r.b2 = 3 * r.p2 + (r.act2 ? r.role : 0);
    r.src1 = r.role == 0 ? lane + 2 : (r.role == 2 ? lane - 2 : lane);
    r.src2 = r.role == 1 ? lane + 1 : (r.role == 2 ? lane - 1 : lane);
    r.bf = t / N2;
    r.kb = t - r.bf * N2;
    r.act3 = r.bf < NLF;
    r.bfc = r.act3 ? r.bf : NLF - 1;
    r.partner = (lane - r.kb) + ((N2 - r.kb) & (N2 - 1));
    r.p3 = r.bfc / 6;
    const int rem3 = r.bfc - 6 * r.p3;
    r.role3 = rem3 >> 1;
    r.j3 = rem3 & 1;
    return r;
}

// The emission steps of y-chunk cy (csteps steps each): u-plane t and v-plane t-1 for
// t = ta..tb-1.  The CTA runs it = it0..tb-1, it0 = -1 in the bottom chunk (step "0a"),
// ta - 1 otherwise (a step that only fills the history).
__host__ __device__ inline void xmarch_chunk(int cy, int csteps, int nyu, int& it0, int& ta, int& tb) {
    ta = 1 + cy * csteps;
    tb = ta + csteps < nyu ? ta + csteps : nyu;
    it0 = cy == 0 ? -1 : ta - 1;
}

// What step it of a CTA transforms and produces.  The inverse lines carry u, w of u-plane
// tu and v of v-plane va, or (combo) the y-interpolation of v-planes va and vb in spectral
// space: combo = -1 for the bottom ghost centre (u-plane 0, step "0a"), +1 for the top one
// (u-plane nyu-1, which has no v-plane tu).  emit: the products of u-plane tu, with v at its
// centre from the new v and the previous step's (weights vca/vcb[vc]) or, vc = -1, the new
// v as it is; emit_v: the products of v-plane tu-1, with u and w at its face from the new
// and the previous step's (weights ufa/ufb[tu-1]).
struct XMStep {
    int tu, va, vb, combo, vc;
    bool emit, emit_v;
};

__host__ __device__ inline XMStep xmarch_step(int it, int ta, int nyu) {
    XMStep s;
    s.emit = it == -1 || it >= ta;
    s.tu = it < 0 ? 0 : it;
    s.va = s.vb = s.tu;
    s.combo = 0;
    if (it == -1) { s.combo = -1; s.va = 1; s.vb = 0; }
    else if (it == nyu - 1) { s.combo = 1; s.va = it - 1; s.vb = it - 2; }
    s.emit_v = s.emit && it >= 1;
    s.vc = (s.emit && it >= 1 && it <= nyu - 2) ? it : -1;
    return s;
}

}  // namespace cfd
