// Host check of the x-face carry of the RK4 stage march (test_flux_carry.py):
// the right-hand side of every cell of a small random periodic grid computed
// by pf::rhs_core in full, and in a march along x that takes each cell's
// x-minus terms from the x-plus terms of the cell before it, must agree bit
// for bit in FP64 and FP32.  Prints the mismatch counts; exit status 1 on any.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pf_flux.cuh"

template <typename T>
struct HostSrc {
    const std::vector<T>*U, *V, *W;
    int n0, n1, n2, i, j, k;
    static int wrap(int a, int n) { return ((a % n) + n) % n; }
    T at(const std::vector<T>& f, int di, int dj, int dk) const {
        return f[((long)wrap(i + di, n0) * n1 + wrap(j + dj, n1)) * n2 + wrap(k + dk, n2)];
    }
    T u(int a, int b, int c) const { return at(*U, a, b, c); }
    T v(int a, int b, int c) const { return at(*V, a, b, c); }
    T w(int a, int b, int c) const { return at(*W, a, b, c); }
    T visc(int, int, int) const { return T(0); }
    T sfs(int, int, int, int) const { return T(0); }
};

template <typename T>
static int mismatches(int n0, int n1, int n2, unsigned seed) {
    std::vector<T> U((size_t)n0 * n1 * n2), V(U.size()), W(U.size());
    srand(seed);
    for (auto* f : {&U, &V, &W})
        for (auto& x : *f) x = T(rand() / double(RAND_MAX) - 0.5);
    const T mu = T(0.01), rho = T(1.3), dxi = T(1.1), dyi = T(0.9), dzi = T(1.7);
    int bad = 0;
    for (int j = 0; j < n1; ++j)
        for (int k = 0; k < n2; ++k) {
            pf::XFace<T> xf;
            for (int i = 0; i < n0; ++i) {
                HostSrc<T> S{&U, &V, &W, n0, n1, n2, i, j, k};
                T a0, a1, a2, b0, b1, b2;
                pf::rhs_core<T, false>(S, mu, rho, dxi, dyi, dzi, false, false, a0, a1, a2);
                if (i == 0)
                    pf::rhs_core<T, false>(S, mu, rho, dxi, dyi, dzi, false, false, b0, b1, b2,
                                           nullptr, &xf);
                else
                    pf::rhs_core<T, true>(S, mu, rho, dxi, dyi, dzi, false, false, b0, b1, b2,
                                          &xf, &xf);
                if (a0 != b0 || a1 != b1 || a2 != b2) ++bad;
            }
        }
    return bad;
}

int main() {
    const int d = mismatches<double>(9, 5, 6, 3) + mismatches<double>(4, 7, 3, 5);
    const int f = mismatches<float>(9, 5, 6, 3) + mismatches<float>(4, 7, 3, 5);
    printf("mismatches fp64 %d fp32 %d\n", d, f);
    return (d || f) ? 1 : 0;
}
