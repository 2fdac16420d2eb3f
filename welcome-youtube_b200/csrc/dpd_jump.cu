// dpd_jump.cu -- jumping ahead in the xoshiro256** stream of the catalyst
// chemistry (host side).
//
// The state transition T of xoshiro256** is linear over GF(2), so T satisfies
// its characteristic polynomial P (degree 256): T^n = (x^n mod P)(T).  P is the
// minimal polynomial of any output bit sequence of the generator; it is found
// once with the Berlekamp-Massey algorithm over 512 bits of the lowest bit of
// s[0].  A jump by n is then x^n mod P by square-and-multiply, applied to a
// state as the XOR of T^i s over the coefficients i that are set.  The device
// uses a table of x^(64 m) mod P (m = 0, 1, ...) to start each 64-draw block
// of a check's stream at its own place (dpd_catalyst.cu, k_cat_stream).
#include <cstring>
#include <mutex>
#include <vector>

#include "dpd_internal.h"

namespace {

void xo_step(uint64_t s[4]) {
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
}

struct Res {  // a residue mod P: bit i of w is the coefficient of x^i (degree < 256)
    uint64_t w[4];
};

uint64_t g_low[4];  // P(x) - x^256
int g_degree = 0;

void find_poly() {
    static std::once_flag once;
    std::call_once(once, [] {
        uint64_t s[4] = {0x9e3779b97f4a7c15ull, 0xbf58476d1ce4e5b9ull, 0x94d049bb133111ebull, 0x2545f4914f6cdd1dull};
        const int N = 512;
        std::vector<int> seq(N), C(N + 1, 0), B(N + 1, 0), T;
        for (int k = 0; k < N; k++) {
            seq[k] = (int)(s[0] & 1);
            xo_step(s);
        }
        C[0] = B[0] = 1;
        int L = 0, m = 1;
        for (int n = 0; n < N; n++) {
            int d = seq[n];
            for (int i = 1; i <= L; i++) d ^= C[i] & seq[n - i];
            if (!d) {
                m++;
                continue;
            }
            T = C;
            for (int i = 0; i + m <= N; i++) C[i + m] ^= B[i];
            if (2 * L <= n) {
                L = n + 1 - L;
                B = T;
                m = 1;
            } else {
                m++;
            }
        }
        // s_n = sum_{i=1..L} c_i s_{n-i}:  P(x) = x^L + sum_i c_i x^(L-i)
        std::memset(g_low, 0, sizeof g_low);
        for (int i = 1; i <= L; i++)
            if (C[i]) {
                const int e = L - i;
                g_low[e >> 6] |= 1ull << (e & 63);
            }
        g_degree = L;
    });
}

Res mulx(Res r) {  // r x mod P
    const uint64_t top = r.w[3] >> 63;
    r.w[3] = (r.w[3] << 1) | (r.w[2] >> 63);
    r.w[2] = (r.w[2] << 1) | (r.w[1] >> 63);
    r.w[1] = (r.w[1] << 1) | (r.w[0] >> 63);
    r.w[0] <<= 1;
    if (top)
        for (int k = 0; k < 4; k++) r.w[k] ^= g_low[k];
    return r;
}

Res mulmod(const Res &a, const Res &b) {  // Horner over the bits of b
    Res r{};
    for (int i = 255; i >= 0; i--) {
        r = mulx(r);
        if ((b.w[i >> 6] >> (i & 63)) & 1)
            for (int k = 0; k < 4; k++) r.w[k] ^= a.w[k];
    }
    return r;
}

Res xpow(uint64_t n) {  // x^n mod P
    Res r{};
    r.w[0] = 1;
    for (int i = 63; i >= 0; i--) {
        r = mulmod(r, r);
        if ((n >> i) & 1) r = mulx(r);
    }
    return r;
}

void apply(const Res &j, const uint64_t s[4], uint64_t out[4]) {  // (j)(T) s
    uint64_t t[4] = {s[0], s[1], s[2], s[3]}, acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 256; i++) {
        if ((j.w[i >> 6] >> (i & 63)) & 1)
            for (int k = 0; k < 4; k++) acc[k] ^= t[k];
        xo_step(t);
    }
    std::memcpy(out, acc, sizeof acc);
}

}  // namespace

// x^(64 m) mod P for m < nblk, 4 words each
int jump_table(int nblk, std::vector<uint64_t> &out) {
    find_poly();
    if (g_degree != 256) return -1;
    out.assign((size_t)nblk * 4, 0);
    Res r{};
    r.w[0] = 1;
    for (int m = 0; m < nblk; m++) {
        std::memcpy(&out[(size_t)m * 4], r.w, sizeof r.w);
        for (int k = 0; k < 64; k++) r = mulx(r);
    }
    return 0;
}

extern "C" int dpd_xoshiro_jump(const uint64_t *state, uint64_t n, uint64_t *out) {
    if (!state || !out) return DPD_E_ARG;
    find_poly();
    if (g_degree != 256) return DPD_E_STATE;
    apply(xpow(n), state, out);
    return DPD_OK;
}
