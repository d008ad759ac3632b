// Host-side check of the register DFTs of cfd_b200/csrc/fft_reg.cuh (compiled by nvcc as
// host code, run on the CPU by tests/test_fft_prune.py).
//
// rdft_z<N1, SIGN, ZM> skips the additions with the inputs that the mask ZM flags as zero;
// the x-line kernel calls it with gap_blocks<N1, N2, N/3>(), the stride-N2 subsequences
// that lie wholly in the 2/3-rule gap.  For every production length and both signs this
// program fills the unmasked inputs with seeded values, the masked ones with zeros, and
// compares rdft_z with rdft element by element: equal values, where a zero may differ
// only in its sign (x + 0 turns -0 into +0, which the pruned path does not do).
// Prints one line per case and exits non-zero on a mismatch.
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "../cfd_b200/csrc/fft_reg.cuh"

using namespace cfd;

static uint64_t g_state = 0x9E3779B97F4A7C15ull;
static double next_uniform() {
    g_state ^= g_state << 13;
    g_state ^= g_state >> 7;
    g_state ^= g_state << 17;
    return (double)(g_state >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

template <typename T2> static bool same(decltype(T2::x) a, decltype(T2::x) b) {
    return a == b || (std::isnan(a) && std::isnan(b));
}

template <typename T2, int N1, int N2, int SIGN> static int check_one(const char* tname) {
    constexpr int N = N1 * N2;
    constexpr unsigned long long ZM = gap_blocks<N1, N2, N / 3>();
    int bad = 0, signed_zero = 0;
    for (int trial = 0; trial < 8; ++trial) {
        T2 a[N1], b[N1];
        for (int n = 0; n < N1; ++n) {
            const bool zero = (ZM >> n) & 1ull;
            // trial 1 puts negative zeros into the live inputs as well
            const double re = zero ? 0.0 : (trial == 1 && n % 3 == 0 ? -0.0 : next_uniform());
            const double im = zero ? 0.0 : (trial == 1 && n % 2 == 0 ? -0.0 : next_uniform());
            a[n] = cx<T2>((decltype(T2::x))re, (decltype(T2::x))im);
            b[n] = a[n];
        }
        rdft<N1, SIGN>(a);
        rdft_z<N1, SIGN, ZM>(b);
        for (int n = 0; n < N1; ++n) {
            if (!same<T2>(a[n].x, b[n].x) || !same<T2>(a[n].y, b[n].y)) ++bad;
            if ((a[n].x == 0 && std::signbit(a[n].x) != std::signbit(b[n].x)) ||
                (a[n].y == 0 && std::signbit(a[n].y) != std::signbit(b[n].y)))
                ++signed_zero;
        }
    }
    std::printf("%s N=%d (%dx%d) sign=%+d mask=%#llx mismatches=%d zero-sign-differences=%d\n", tname, N, N1, N2,
                SIGN, ZM, bad, signed_zero);
    return bad;
}

template <typename T2, int N1, int N2> static int check_len(const char* tname) {
    return check_one<T2, N1, N2, +1>(tname) + check_one<T2, N1, N2, -1>(tname);
}

template <typename T2> static int check_all(const char* tname) {
    int bad = 0;
    bad += check_len<T2, 8, 8>(tname);
    bad += check_len<T2, 8, 12>(tname);
    bad += check_len<T2, 8, 16>(tname);
    bad += check_len<T2, 16, 12>(tname);
    bad += check_len<T2, 16, 24>(tname);
    bad += check_len<T2, 32, 24>(tname);
    // the transposed splits (cfd_tuning xsplit = 2)
    bad += check_len<T2, 16, 4>(tname);
    bad += check_len<T2, 12, 8>(tname);
    bad += check_len<T2, 16, 8>(tname);
    bad += check_len<T2, 12, 16>(tname);
    bad += check_len<T2, 24, 16>(tname);
    bad += check_len<T2, 24, 32>(tname);
    return bad;
}

int main() {
    const int bad = check_all<float2>("float2") + check_all<double2>("double2");
    std::printf("%s\n", bad ? "FAIL" : "OK");
    return bad ? 1 : 0;
}
