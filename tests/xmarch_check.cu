// Host-side check of the launch geometry, thread roles and y-step sequence of the x-line
// pass marching in y (cfd_b200/csrc/xmarch_plan.cuh; compiled by nvcc as host code and run
// on the CPU by tests/test_xmarch_plan.py).
//
// For every split the kernel is built for and 2 and 4 rows per CTA: every shared-memory
// index of the three phases lies inside its buffer, every work item of a phase is taken by
// exactly one thread, the physical phase reads back exactly the inverse exchange cells the
// first step wrote and the last step reads exactly the forward cells the physical phase
// wrote, shuffle sources are the intended lanes of the same warp, and the unpack covers
// kx = 0..N/3 once with the partner holding X_N-k.  For many channel heights and y-chunk
// lengths: every u-plane and v-plane is produced exactly once, each from the planes whose
// values the interpolation needs (the new step's and the previous step's).
// Prints one line per case and "OK", and exits non-zero on the first failure.
#include <cstdio>
#include <cstdlib>
#include <set>
#include <tuple>
#include <vector>

#include "../cfd_b200/csrc/xmarch_plan.cuh"

using namespace cfd;

#define REQUIRE(c, ...)                                        \
    do {                                                       \
        if (!(c)) {                                            \
            std::printf("FAIL %s:%d: ", __FILE__, __LINE__);   \
            std::printf(__VA_ARGS__);                          \
            std::printf("\n");                                 \
            std::exit(1);                                      \
        }                                                      \
    } while (0)

static void check_roles(int N1, int N2, int RW) {
    const int N = N1 * N2, HX = N / 3, KA = HX / N2 + 1;
    const int NT = xmarch_threads(N1, N2, RW);
    const int pairs = RW / 2, NLI = 3 * pairs, NLF = 6 * pairs, NTRI = pairs * N1;
    const long long L1 = xmarch_l1(N1, N2), L2 = xmarch_l2(N1, N2);
    REQUIRE(NT % 32 == 0 && NT <= 256, "NT %d", NT);
    REQUIRE(L1 >= (long long)N1 * (N2 + 1) && L2 >= (long long)N2 * (N1 + 1), "pitches");
    REQUIRE(xmarch_smem_elems(N1, N2, RW) ==
                NLI * L1 + NLF * L2 + (long long)N2 * NT + (long long)N1 * (N2 + 1), "smem");
    std::vector<XMRoles> r(NT);
    for (int t = 0; t < NT; ++t) r[t] = xmarch_roles(t, RW, N1, N2);

    // step 1: (line, column) once each; writes of the inverse exchange
    std::set<std::tuple<int, int>> items;
    std::set<long long> exi_w;
    for (int t = 0; t < NT; ++t) {
        if (!r[t].act1) continue;
        REQUIRE(r[t].b1 < NLI && r[t].n2 < N2 && r[t].p1 < pairs && r[t].role1 < 3, "step 1 role of %d", t);
        REQUIRE(items.insert({r[t].b1, r[t].n2}).second, "step 1 item twice");
        for (int q = 0; q < N1; ++q) {
            const long long i = r[t].b1 * L1 + q * (N2 + 1) + r[t].n2;
            REQUIRE(i >= 0 && i < NLI * L1, "exi write %lld", i);
            REQUIRE(exi_w.insert(i).second, "exi cell written twice");
        }
    }
    REQUIRE((int)items.size() == NLI * N2, "step 1 covers %zu of %d", items.size(), NLI * N2);

    // physical phase: triples once each; reads of the inverse exchange, shuffle sources,
    // writes of the forward exchange
    std::set<std::tuple<int, int, int>> tri;
    std::set<long long> exi_r, exf_w;
    for (int t = 0; t < NT; ++t) {
        const XMRoles& a = r[t];
        // every lane takes part in the reads (inactive ones on line 0, column 0)
        for (int q = 0; q < N2; ++q) {
            const long long i = a.b2 * L1 + a.k1 * (N2 + 1) + q;
            REQUIRE(i >= 0 && i < NLI * L1, "exi read %lld", i);
            if (a.act2) exi_r.insert(i);
        }
        if (!a.act2) continue;
        REQUIRE(a.p2 < pairs && a.k1 < N1 && a.role < 3 && a.b2 == 3 * a.p2 + a.role, "triple role of %d", t);
        REQUIRE(tri.insert({a.p2, a.k1, a.role}).second, "triple lane twice");
        const int lane = t & 31, wbase = t & ~31;
        auto same_triple = [&](int src, int want_role) {
            REQUIRE(src >= 0 && src < 32 && wbase + src < NT, "shuffle source %d of lane %d", src, lane);
            const XMRoles& b = r[wbase + src];
            REQUIRE(b.act2 && b.p2 == a.p2 && b.k1 == a.k1 && b.role == want_role, "shuffle partner of %d", t);
        };
        if (a.role == 0) same_triple(a.src1, 2);          // A reads the face w of C
        if (a.role == 1) same_triple(a.src2, 2);          // B reads the face w' of C
        if (a.role == 2) { same_triple(a.src1, 0); same_triple(a.src2, 1); }  // C reads u, u'
        for (int j = 0; j < 2; ++j)
            for (int q = 0; q < N2; ++q) {
                const long long i = (long long)(6 * a.p2 + 2 * a.role + j) * L2 + q * (N1 + 1) + a.k1;
                REQUIRE(i >= 0 && i < NLF * L2, "exf write %lld", i);
                REQUIRE(exf_w.insert(i).second, "exf cell written twice");
            }
    }
    REQUIRE((int)tri.size() == 3 * NTRI, "triples cover %zu of %d", tri.size(), 3 * NTRI);
    REQUIRE(exi_r == exi_w, "the physical phase does not read what step 1 wrote");

    // step 2': (forward line, column) once each; reads of the forward exchange; partners
    std::set<std::tuple<int, int>> f_items;
    std::set<long long> exf_r;
    for (int t = 0; t < NT; ++t) {
        const XMRoles& a = r[t];
        REQUIRE(a.bfc < NLF && a.p3 < pairs && a.role3 < 3 && a.j3 < 2 &&
                    a.bfc == 6 * a.p3 + 2 * a.role3 + a.j3, "step 2' line of %d", t);
        for (int q = 0; q < N1; ++q) {
            const long long i = a.bfc * L2 + a.kb * (N1 + 1) + q;
            REQUIRE(i >= 0 && i < NLF * L2, "exf read %lld", i);
            if (a.act3) exf_r.insert(i);
        }
        const int wbase = t & ~31;
        REQUIRE(a.partner >= 0 && a.partner < 32 && wbase + a.partner < NT, "partner lane of %d", t);
        const XMRoles& b = r[wbase + a.partner];
        REQUIRE(b.bf == a.bf && b.kb == (N2 - a.kb) % N2, "partner of %d holds kb %d of line %d", t, b.kb, b.bf);
        if (!a.act3) continue;
        REQUIRE(f_items.insert({a.bf, a.kb}).second, "step 2' item twice");
    }
    REQUIRE((int)f_items.size() == NLF * N2, "step 2' covers %zu of %d", f_items.size(), NLF * N2);
    REQUIRE(exf_r == exf_w, "the last step does not read what the physical phase wrote");

    // unpack: k = kb + N2 ka <= HX once each, X_N-k at element ka' of lane N2 - kb
    std::vector<int> seen(HX + 1, 0);
    for (int kb = 0; kb < N2; ++kb)
        for (int ka = 0; ka < KA; ++ka) {
            const int k = kb + N2 * ka;
            if (k > HX) continue;
            ++seen[k];
            const int kbp = (N2 - kb) % N2, kap = kb == 0 ? (N1 - ka) % N1 : N1 - 1 - ka;
            REQUIRE(kap >= 0 && kap < N1 && (kbp + N2 * kap) % N == (N - k) % N, "partner element of k %d", k);
        }
    for (int k = 0; k <= HX; ++k) REQUIRE(seen[k] == 1, "kx %d unpacked %d times", k, seen[k]);
    std::printf("roles %dx%d rows %d: %d threads, %lld elements of shared memory\n", N1, N2, RW, NT,
                xmarch_smem_elems(N1, N2, RW));
}

// The sequence of steps over all y-chunks of a channel with nyu u-planes (nyu - 1 v-planes).
static void check_steps(int nyu, int csteps) {
    const int nch = (nyu - 1 + csteps - 1) / csteps;
    std::vector<int> nu(nyu, 0), nv(nyu - 1, 0);
    for (int cy = 0; cy < nch; ++cy) {
        int it0, ta, tb;
        xmarch_chunk(cy, csteps, nyu, it0, ta, tb);
        REQUIRE(ta >= 1 && ta < tb && tb <= nyu && it0 == (cy == 0 ? -1 : ta - 1), "chunk %d of nyu %d", cy, nyu);
        int hu = -2, hv = -2;  // the planes of the previous step's u, w and v (-2: none, -3: a ghost v)
        for (int it = it0; it < tb; ++it) {
            const XMStep s = xmarch_step(it, ta, nyu);
            REQUIRE(s.tu >= 0 && s.tu < nyu, "u-plane %d", s.tu);
            REQUIRE(s.va >= 0 && s.va <= nyu - 2 && s.vb >= 0 && s.vb <= nyu - 2, "v-planes %d %d", s.va, s.vb);
            if (s.combo == -1) REQUIRE(it == -1 && s.tu == 0 && s.va == 1 && s.vb == 0, "bottom ghost");
            if (s.combo == 1) REQUIRE(it == nyu - 1 && s.va == nyu - 2 && s.vb == nyu - 3, "top ghost");
            if (s.combo == 0) REQUIRE(s.va == s.tu, "v-plane %d with u-plane %d", s.va, s.tu);
            REQUIRE(s.emit == (it == -1 || it >= ta), "emit at %d", it);
            if (s.emit) {
                ++nu[s.tu];
                if (s.vc >= 0) {  // v at the centre from the new v-plane tu and the previous tu-1
                    REQUIRE(s.vc == s.tu && s.combo == 0 && hv == s.tu - 1, "centre of u-plane %d", s.tu);
                } else {          // a ghost centre: the new v is already interpolated
                    REQUIRE((s.tu == 0 && s.combo == -1) || (s.tu == nyu - 1 && s.combo == 1), "ghost %d", s.tu);
                }
            }
            if (s.emit_v) {       // v-plane tu-1: u, w of u-planes tu (new) and tu-1, v of v-plane tu-1
                REQUIRE(s.emit && s.tu >= 1 && hu == s.tu - 1 && hv == s.tu - 1, "face of v-plane %d", s.tu - 1);
                ++nv[s.tu - 1];
            }
            hu = s.tu;
            hv = s.combo == 0 ? s.va : -3;
        }
    }
    for (int j = 0; j < nyu; ++j) REQUIRE(nu[j] == 1, "u-plane %d of %d produced %d times", j, nyu, nu[j]);
    for (int j = 0; j < nyu - 1; ++j) REQUIRE(nv[j] == 1, "v-plane %d of %d produced %d times", j, nyu - 1, nv[j]);
}

int main() {
    const int splits[5][2] = {{8, 8}, {12, 8}, {8, 16}, {12, 16}, {24, 16}};
    for (auto& s : splits)
        for (int rw : {2, 4}) check_roles(s[0], s[1], rw);
    int cases = 0;
    for (int nyu = 4; nyu <= 70; ++nyu)
        for (int c : {2, 3, 4, 5, 6, 8, 12, 16, 32, 100}) { check_steps(nyu, c); ++cases; }
    for (int nyu : {98, 154, 176, 238, 284, 348, 386})
        for (int c : {2, 4, 6, 8, 12, 16, 20, 32, 64}) { check_steps(nyu, c); ++cases; }
    std::printf("steps: %d channel heights and y-chunk lengths\n", cases);
    std::printf("OK\n");
    return 0;
}
