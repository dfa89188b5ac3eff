// Host check of the RK4 stage's face reuse (test_flux_carry.py): the
// right-hand side of every cell of a small random periodic grid computed by
// pf::rhs_core in full must agree bit for bit, in FP64 and FP32, with (1) a
// march along x that takes each cell's x-minus terms from the x-plus terms of
// the cell before it, and (2) the face form that assembles each cell from the
// plus-face terms of the cell and of its neighbours at i-1, j-1, k-1.  Prints
// the mismatch counts; exit status 1 on any.
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

// The face form: every cell assembled from its own plus-face terms and the
// plus-face terms of its neighbours at i-1, j-1, k-1 (pf::plus_faces,
// pf::assemble_faces) against pf::rhs_core.
template <typename T>
static int face_mismatches(int n0, int n1, int n2, unsigned seed) {
    std::vector<T> U((size_t)n0 * n1 * n2), V(U.size()), W(U.size());
    srand(seed);
    for (auto* f : {&U, &V, &W})
        for (auto& x : *f) x = T(rand() / double(RAND_MAX) - 0.5);
    const T mu = T(0.013), rho = T(0.7), dxi = T(1.3), dyi = T(0.8), dzi = T(2.1);
    const pf::FluxCoef<T> c = pf::flux_coef<T>(mu, rho, dxi, dyi, dzi);
    int bad = 0;
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k) {
                HostSrc<T> S{&U, &V, &W, n0, n1, n2, i, j, k};
                T a0, a1, a2, b0, b1, b2;
                pf::rhs_core<T, false>(S, mu, rho, dxi, dyi, dzi, false, false, a0, a1, a2);
                const pf::PlusFaces<T> p = pf::plus_faces<T>(S, c);
                const pf::Shifted<HostSrc<T>> sx{S, -1, 0, 0}, sy{S, 0, -1, 0}, sz{S, 0, 0, -1};
                const auto xm = pf::plus_faces<T, true, false, false>(sx, c).x;
                const auto ym = pf::plus_faces<T, false, true, false>(sy, c).y;
                const auto zm = pf::plus_faces<T, false, false, true>(sz, c).z;
                pf::assemble_faces(p, xm, ym, zm, c, b0, b1, b2);
                if (a0 != b0 || a1 != b1 || a2 != b2) ++bad;
            }
    return bad;
}

int main() {
    const int d = mismatches<double>(9, 5, 6, 3) + mismatches<double>(4, 7, 3, 5);
    const int f = mismatches<float>(9, 5, 6, 3) + mismatches<float>(4, 7, 3, 5);
    printf("mismatches fp64 %d fp32 %d\n", d, f);
    const int fd = face_mismatches<double>(7, 6, 5, 11) + face_mismatches<double>(3, 4, 9, 12);
    const int ff = face_mismatches<float>(7, 6, 5, 11) + face_mismatches<float>(3, 4, 9, 12);
    printf("face mismatches fp64 %d fp32 %d\n", fd, ff);
    return (d || f || fd || ff) ? 1 : 0;
}
