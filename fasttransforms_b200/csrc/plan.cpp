// Host-side plan generation: rotation tables, dense connection matrices and
// the longest-first task lists of the rotation kernel.
//
// The connection matrices are the reference's: generalised eigenvectors of
// upper-triangular banded pencils (A, B), computed in long double and rounded
// to double (src/transforms.c:50-108, src/banded_source.c:779-800).  The
// operators and the recurrences keep the reference's expression order so the
// rounded matrices agree with the reference's bit for bit.  The only change is
// the evaluation schedule: columns are independent, so they are computed by a
// pool of host threads, each column into its own long-double buffer (no n x n
// long-double matrix).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "ft_internal.h"

namespace ftb {

// ---------------------------------------------------------------------------
// Rotation tables (FP64 square roots of rationals).
// sph: src/rotations.c:116-133, tri: :143-160, disk: :173-190 (negated sine),
// rect: :270-287 (the sph packing, entries depending on beta).
// ---------------------------------------------------------------------------
void rotation_tables(int kind, int n, double alpha, double beta, double gamma, double * s, double * c) {
    if (kind == SPH) {
        for (int m = 0; m < n; m++)
            for (int l = 0; l < n - m; l++) {
                const double nums = (double) ((long long) (l + 1) * (l + 2));   // exact integers (no int overflow)
                const double numc = (double) ((long long) (2 * m + 2) * (2 * l + 2 * m + 5));
                const double den = (double) ((long long) (l + 2 * m + 3) * (l + 2 * m + 4));
                const long long o = Geo::table_base(SPH, n, m) + l;
                s[o] = std::sqrt(nums / den);
                c[o] = std::sqrt(numc / den);
            }
    } else if (kind == TRI) {
        for (int m = 0; m < n; m++)
            for (int l = 0; l < n - m; l++) {
                const double nums = (l + 1) * (l + alpha + 1);
                const double numc = (2 * m + beta + gamma + 2) * (2 * l + 2 * m + alpha + beta + gamma + 4);
                const double den = (l + 2 * m + beta + gamma + 3) * (l + 2 * m + alpha + beta + gamma + 3);
                const long long o = Geo::table_base(TRI, n, m) + l;
                s[o] = std::sqrt(nums / den);
                c[o] = std::sqrt(numc / den);
            }
    } else if (kind == RECT) {
        for (int m = 0; m < n; m++)
            for (int l = 0; l < n - m; l++) {
                const double nums = (l + 1) * (l + 2);
                const double numc = (2 * m + 2 * beta + 3) * (2 * l + 2 * m + 2 * beta + 6);
                const double den = (l + 2 * m + 2 * beta + 4) * (l + 2 * m + 2 * beta + 5);
                const long long o = Geo::table_base(RECT, n, m) + l;
                s[o] = std::sqrt(nums / den);
                c[o] = std::sqrt(numc / den);
            }
    } else {
        for (int m = 0; m < 2 * n - 1; m++)
            for (int l = 0; l < n - (m + 1) / 2; l++) {
                const double nums = (l + 1) * (l + beta + 1);
                const double numc = (m + alpha + 1) * (2 * l + m + alpha + beta + 3);
                const double den = (l + m + alpha + 2) * (l + m + alpha + beta + 2);
                const long long o = Geo::table_base(DISK, n, m) + l;
                s[o] = -std::sqrt(nums / den);
                c[o] = std::sqrt(numc / den);
            }
    }
}

// ---------------------------------------------------------------------------
// Banded operators in long double.  Entry (i, j) is stored for -l <= j-i <= u.
// ---------------------------------------------------------------------------
namespace {

typedef long double ld;
const ld kEps = 0x1p-64L;   // src/ftinternal.h:83
const ld ONE = 1, TWO = 2;

struct Banded {
    int n, l, u;
    std::vector<ld> d;
    Banded(int n_, int l_, int u_) : n(n_), l(l_), u(u_), d((size_t) n_ * (l_ + u_ + 1), 0.0L) {}
    ld get(int i, int j) const {
        if (0 <= i && 0 <= j && -l <= j - i && j - i <= u && i < n && j < n)
            return d[(size_t) (u + i - j) + (size_t) j * (l + u + 1)];
        return 0;
    }
    void set(ld v, int i, int j) {
        if (0 <= i && 0 <= j && -l <= j - i && j - i <= u && i < n && j < n)
            d[(size_t) (u + i - j) + (size_t) j * (l + u + 1)] = v;
    }
};

// C <- alpha*A*B + beta*C   (src/banded_source.c:288-305)
void gbmm(ld alpha, const Banded & A, const Banded & B, ld beta, Banded & C) {
    const int n = A.n;
    for (int j = 0; j < n; j++)
        for (int i = std::max(0, j - C.u); i < std::min(n, j + C.l + 1); i++) {
            ld ab = 0;
            for (int k = std::max(std::max(0, i - A.l), j - B.u); k < std::min(std::min(n, i + A.u + 1), j + B.l + 1); k++)
                ab += A.get(i, k) * B.get(k, j);
            const ld c = C.get(i, j);
            C.set(alpha * ab + beta * c, i, j);
        }
}

// C <- alpha*A + beta*B   (src/banded_source.c:333-343)
void banded_add(ld alpha, const Banded & A, ld beta, const Banded & B, Banded & C) {
    const int n = C.n;
    for (int j = 0; j < n; j++)
        for (int i = std::max(0, j - C.u); i < std::min(n, j + C.l + 1); i++)
            C.set(alpha * A.get(i, j) + beta * B.get(i, j), i, j);
}

// Eigenvectors of the pencil, one column at a time (src/banded_source.c:779-800).
// diag[j] is V(j, j); the result is rounded to double into V (n x n, column-major).
double * eigenvectors(const Banded & A, const Banded & B, const std::vector<ld> & diag) {
    const int n = A.n;
    const int b = std::max(A.u, B.u);
    double * V = static_cast<double *>(std::calloc((size_t) n * n + 1, sizeof(double)));
    if (!V) return nullptr;
    // the pencil's bands, flattened for the inner loop
    std::vector<ld> Ad((size_t) n * (b + 1)), Bd((size_t) n * (b + 1));
    for (int i = 0; i < n; i++)
        for (int o = 0; o <= b; o++) {
            Ad[(size_t) i * (b + 1) + o] = A.get(i, i + o);
            Bd[(size_t) i * (b + 1) + o] = B.get(i, i + o);
        }
    auto column = [&](int j, std::vector<ld> & v) {
        v[j] = diag[j];
        const ld lam = Ad[(size_t) j * (b + 1)] / Bd[(size_t) j * (b + 1)];
        for (int i = j - 1; i >= 0; i--) {
            ld t = 0, kt = 0;
            const int kend = std::min(i + b + 1, n);
            for (int k = i + 1; k < kend; k++) {
                const ld a = Ad[(size_t) i * (b + 1) + (k - i)], bb = Bd[(size_t) i * (b + 1) + (k - i)];
                t += (a - lam * bb) * v[k];
                kt += (std::fabs(a) + std::fabs(lam * bb)) * std::fabs(v[k]);
            }
            const ld aii = Ad[(size_t) i * (b + 1)], bii = Bd[(size_t) i * (b + 1)];
            const ld d = lam * bii - aii;
            const ld kd = std::fabs(lam * bii) + std::fabs(aii);
            if (std::fabs(d) < 4 * kd * kEps || std::fabs(t) < 4 * kt * kEps)
                v[i] = 0;
            else
                v[i] = t / d;
        }
        double * out = V + (size_t) j * n;
        for (int i = 0; i <= j; i++) out[i] = (double) v[i];
    };
    if (n > 0) V[0] = (double) diag[0];
    const int set = host_threads();   // ft_set_num_threads, 0: unset
    unsigned nt = set > 0 ? (unsigned) set : std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 256) nt = 1;
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nt; w++)
        pool.emplace_back([&, w]() {
            std::vector<ld> v(n);
            // interleave columns so every worker gets a similar share of the O(j) work
            for (int j = 1 + (int) w; j < n; j += (int) nt) column(j, v);
        });
    for (auto & th : pool) th.join();
    return V;
}

}  // namespace

// src/banded_source.c:2316-2338 (A, B) and :2024-2061 (diagonal); src/transforms.c:50-63
double * connection_legendre_to_chebyshev(int normleg, int normcheb, int n) {
    Banded A(n, 0, 2), B(n, 0, 2);
    if (n > 1) A.set(2, 1, 1);
    for (int i = 2; i < n; i++) {
        A.set(-i * (i - ONE), i - 2, i);
        A.set(i * (i + ONE), i, i);
    }
    if (n > 0) B.set(normcheb ? std::sqrt((ld) 2) : 2, 0, 0);
    if (n > 1) B.set(1, 1, 1);
    for (int i = 2; i < n; i++) {
        B.set(-1, i - 2, i);
        B.set(1, i, i);
    }
    std::vector<ld> D(n);
    if (normleg) {
        if (normcheb) {
            if (n > 0) D[0] = std::sqrt((ld) 0.5) * std::tgamma((ld) 0.5);
            if (n > 1) D[1] = std::sqrt((ld) 1.5) * D[0];
        } else {
            if (n > 0) D[0] = std::sqrt((ld) 0.5);
            if (n > 1) D[1] = std::sqrt((ld) 1.5);
        }
        for (int i = 2; i < n; i++) D[i] = std::sqrt((2 * i + 1) * (2 * i - ONE)) * D[i - 1] / (2 * i);
    } else {
        if (normcheb) {
            if (n > 0) D[0] = std::tgamma((ld) 0.5);
            if (n > 1) D[1] = D[0] / std::sqrt((ld) 2);
        } else {
            if (n > 0) D[0] = 1;
            if (n > 1) D[1] = 1;
        }
        for (int i = 2; i < n; i++) D[i] = (2 * i - 1) * D[i - 1] / (2 * i);
    }
    return eigenvectors(A, B, D);
}

// src/banded_source.c:2340-2384 (A, B) and :2063-2100 (diagonal); src/transforms.c:65-78
double * connection_chebyshev_to_legendre(int normcheb, int normleg, int n) {
    Banded A(n, 0, 2), B(n, 0, 2);
    if (normleg) {
        if (n > 1) A.set(std::sqrt(TWO / 5), 1, 1);
        for (int i = 2; i < n; i++) {
            A.set(-(i + 1) * std::sqrt(((i - ONE) * i) / ((2 * i - ONE) * (2 * i + 1))) * (i + 1), i - 2, i);
            A.set(i * std::sqrt(((i + ONE) * (i + 2)) / ((2 * i + ONE) * (2 * i + 3))) * i, i, i);
        }
        if (n > 0) B.set(std::sqrt(TWO / 3), 0, 0);
        if (n > 1) B.set(std::sqrt(TWO / 5), 1, 1);
        for (int i = 2; i < n; i++) {
            B.set(-std::sqrt(((i - ONE) * i) / ((2 * i - ONE) * (2 * i + 1))), i - 2, i);
            B.set(std::sqrt(((i + ONE) * (i + 2)) / ((2 * i + ONE) * (2 * i + 3))), i, i);
        }
    } else {
        if (n > 1) A.set(ONE / 3, 1, 1);
        for (int i = 2; i < n; i++) {
            A.set(-(i + 1) / (2 * i + ONE) * (i + 1), i - 2, i);
            A.set(i / (2 * i + ONE) * i, i, i);
        }
        if (n > 0) B.set(1, 0, 0);
        if (n > 1) B.set(ONE / 3, 1, 1);
        for (int i = 2; i < n; i++) {
            B.set(-1 / (2 * i + ONE), i - 2, i);
            B.set(1 / (2 * i + ONE), i, i);
        }
    }
    std::vector<ld> D(n);
    if (normcheb) {
        if (normleg) {
            if (n > 0) D[0] = std::sqrt((ld) 2) / std::tgamma((ld) 0.5);
            if (n > 1) D[1] = D[0] / std::sqrt((ld) 1.5);
            for (int i = 2; i < n; i++) D[i] = (2 * i) / std::sqrt((2 * i + 1) * (2 * i - ONE)) * D[i - 1];
        } else {
            if (n > 0) D[0] = 1 / std::tgamma((ld) 0.5);
            if (n > 1) D[1] = std::sqrt((ld) 2) * D[0];
            for (int i = 2; i < n; i++) D[i] = (2 * i) * D[i - 1] / (2 * i - 1);
        }
    } else {
        if (normleg) {
            if (n > 0) D[0] = std::sqrt((ld) 2);
            if (n > 1) D[1] = 1 / std::sqrt((ld) 1.5);
            for (int i = 2; i < n; i++) D[i] = (2 * i) / std::sqrt((2 * i + 1) * (2 * i - ONE)) * D[i - 1];
        } else {
            if (n > 0) D[0] = 1;
            if (n > 1) D[1] = 1;
            for (int i = 2; i < n; i++) D[i] = (2 * i) * D[i - 1] / (2 * i - 1);
        }
    }
    return eigenvectors(A, B, D);
}

// src/banded_source.c:2386-2430 (A, B) and :2102-2131 (diagonal); src/transforms.c:80-93
double * connection_ultraspherical(int norm1, int norm2, int n, double lambda_d, double mu_d) {
    const ld lambda = lambda_d, mu = mu_d;
    Banded A(n, 0, 2), B(n, 0, 2);
    if (norm2) {
        if (n > 1) A.set((1 + 2 * lambda) * std::copysign(std::sqrt((2 * mu + 1) / (2 * mu + 4)), mu), 1, 1);
        for (int i = 2; i < n; i++) {
            A.set(-(i + 2 * mu) * (i + 2 * (mu - lambda)) * std::copysign(std::sqrt((i * (i - ONE)) / (4 * (i + mu) * (i + mu - 1))), mu), i - 2, i);
            A.set(i * (i + 2 * lambda) * std::copysign(std::sqrt(((i + 2 * mu) * (i + 2 * mu + 1)) / (4 * (i + mu) * (i + mu + 1))), mu), i, i);
        }
        if (n > 0) B.set(std::sqrt((2 * mu + 1) / (2 * mu + 2)), 0, 0);
        if (n > 1) B.set(std::copysign(std::sqrt((2 * mu + 1) / (2 * mu + 4)), mu), 1, 1);
        for (int i = 2; i < n; i++) {
            B.set(-std::copysign(std::sqrt((i * (i - ONE)) / (4 * (i + mu) * (i + mu - 1))), mu), i - 2, i);
            B.set(std::copysign(std::sqrt(((i + 2 * mu) * (i + 2 * mu + 1)) / (4 * (i + mu) * (i + mu + 1))), mu), i, i);
        }
    } else {
        if (n > 1) A.set((1 + 2 * lambda) * mu / (1 + mu), 1, 1);
        for (int i = 2; i < n; i++) {
            A.set(-(i + 2 * mu) * (i + 2 * (mu - lambda)) * mu / (i + mu), i - 2, i);
            A.set(i * (i + 2 * lambda) * mu / (i + mu), i, i);
        }
        if (n > 0) B.set(1, 0, 0);
        if (n > 1) B.set(mu / (1 + mu), 1, 1);
        for (int i = 2; i < n; i++) {
            B.set(-mu / (i + mu), i - 2, i);
            B.set(mu / (i + mu), i, i);
        }
    }
    std::vector<ld> D(n);
    const ld half = 0.5;
    if (norm1) {
        if (norm2) {
            if (n > 0) D[0] = std::sqrt(std::tgamma(lambda + 1) / (std::tgamma(half) * std::tgamma(lambda + half))) * std::sqrt(std::tgamma(half) * std::tgamma(mu + half) / std::tgamma(mu + 1));
            for (int i = 1; i < n; i++)
                D[i] = std::sqrt((i - 1 + mu) / i * (i - 1 + 2 * mu) / (i + mu)) * std::sqrt(i / (i - 1 + lambda) * (i + lambda) / (i - 1 + 2 * lambda)) * (i - 1 + lambda) / (i - 1 + mu) * D[i - 1];
        } else {
            if (n > 0) D[0] = std::sqrt(std::tgamma(lambda + 1) / (std::tgamma(half) * std::tgamma(lambda + half)));
            for (int i = 1; i < n; i++)
                D[i] = std::sqrt(i / (i - 1 + lambda) * (i + lambda) / (i - 1 + 2 * lambda)) * (i - 1 + lambda) / (i - 1 + mu) * D[i - 1];
        }
    } else {
        if (norm2) {
            if (n > 0) D[0] = std::sqrt(std::tgamma(half) * std::tgamma(mu + half) / std::tgamma(mu + 1));
            for (int i = 1; i < n; i++)
                D[i] = std::sqrt((i - 1 + mu) / i * (i - 1 + 2 * mu) / (i + mu)) * (i - 1 + lambda) / (i - 1 + mu) * D[i - 1];
        } else {
            if (n > 0) D[0] = 1;
            for (int i = 1; i < n; i++) D[i] = (i - 1 + lambda) / (i - 1 + mu) * D[i - 1];
        }
    }
    return eigenvectors(A, B, D);
}

namespace {
// Jacobi operators, normalised form (the only one the harmonic planners use).
// derivative: src/banded_source.c:1774-1795
Banded jacobi_derivative(int n, int order, ld alpha, ld beta) {
    Banded A(n, -order, order);
    for (int j = order; j < n; j++) {
        ld v = 1;
        for (int k = 0; k < order; k++) v *= (j - k) * (j + alpha + beta + k + 1);
        v = std::sqrt(v);
        A.set(v, j - order, j);
    }
    return A;
}
// multiplication by x: src/banded_source.c:1797-1841
Banded jacobi_multiplication(int n, ld alpha, ld beta) {
    Banded A(n, 1, 1);
    for (int j = 0; j < n; j++) {
        ld v;
        if (j == 1)
            v = 2 * std::sqrt(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * std::sqrt((j * (j + alpha) * (j + beta) * (j + alpha + beta)) / ((2 * j + alpha + beta - 1) * (2 * j + alpha + beta) * (2 * j + alpha + beta) * (2 * j + alpha + beta + 1)));
        A.set(v, j - 1, j);
        if (j == 0) {
            v = (beta - alpha) / (alpha + beta + 2);
            A.set(v, 0, 0);
            v = 2 * std::sqrt(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 2) * (alpha + beta + 3)));
            A.set(v, 1, 0);
        } else {
            v = ((beta - alpha) * (alpha + beta)) / ((2 * j + alpha + beta) * (2 * j + alpha + beta + 2));
            A.set(v, j, j);
            v = 2 * std::sqrt(((j + 1) * (j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
            A.set(v, j + 1, j);
        }
    }
    return A;
}
// raising: src/banded_source.c:1843-1873
Banded jacobi_raising(int n, ld alpha, ld beta) {
    Banded A(n, 0, 2);
    for (int j = 0; j < n; j++) {
        ld v = -2 * std::sqrt(((j - 1) * j * (j + alpha) * (j + beta)) / ((2 * j + alpha + beta - 1) * (2 * j + alpha + beta) * (2 * j + alpha + beta) * (2 * j + alpha + beta + 1)));
        A.set(v, j - 2, j);
        v = 2 * (alpha - beta) * std::sqrt(j * (j + alpha + beta + 1)) / ((2 * j + alpha + beta) * (2 * j + alpha + beta + 2));
        A.set(v, j - 1, j);
        if (j == 0)
            v = 2 * std::sqrt(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * std::sqrt(((j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
        A.set(v, j, j);
    }
    return A;
}
// lowering: src/banded_source.c:1875-1903
Banded jacobi_lowering(int n, ld alpha, ld beta) {
    Banded A(n, 2, 0);
    for (int j = 0; j < n; j++) {
        ld v;
        if (j == 0)
            v = 2 * std::sqrt(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * std::sqrt(((j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
        A.set(v, j, j);
        v = 2 * (alpha - beta) * std::sqrt((j + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 4));
        A.set(v, j + 1, j);
        v = -2 * std::sqrt(((j + 1) * (j + 2) * (j + alpha + 2) * (j + beta + 2)) / ((2 * j + alpha + beta + 3) * (2 * j + alpha + beta + 4) * (2 * j + alpha + beta + 4) * (2 * j + alpha + beta + 5)));
        A.set(v, j + 2, j);
    }
    return A;
}
}  // namespace

// Normalised Jacobi (alpha, beta) -> (gamma, delta): A = sigma D^2 + tau D
// (src/banded_source.c:2432-2451), B = raising (:2453-2456), diagonal
// (:2133-2142); planner src/transforms.c:95-108 with norm1 = norm2 = 1.
double * connection_jacobi(int n, double alpha_d, double beta_d, double gamma_d, double delta_d) {
    const ld alpha = alpha_d, beta = beta_d, gamma = gamma_d, delta = delta_d;
    Banded A(n, 0, 2);
    {
        const Banded D1 = jacobi_derivative(n, 1, gamma, delta);
        const Banded D2 = jacobi_derivative(n, 2, gamma, delta);
        const Banded L1 = jacobi_lowering(n, gamma + 1, delta + 1);
        const Banded M1 = jacobi_multiplication(n, gamma + 1, delta + 1);
        gbmm(-1, L1, D2, 0, A);
        banded_add(1, A, alpha - beta, D1, A);
        gbmm(alpha + beta + 2, M1, D1, 1, A);
    }
    const Banded B = jacobi_raising(n, gamma, delta);
    std::vector<ld> D(n);
    if (n > 0)
        D[0] = std::sqrt(std::tgamma(alpha + beta + 2) / (std::pow((ld) 2, alpha + beta + 1) * std::tgamma(alpha + 1) * std::tgamma(beta + 1)) * (std::pow((ld) 2, gamma + delta + 1) * std::tgamma(gamma + 1) * std::tgamma(delta + 1)) / std::tgamma(gamma + delta + 2));
    if (n > 1)
        D[1] = (alpha + beta + 2) / (gamma + delta + 2) * std::sqrt((alpha + beta + 3) / ((alpha + 1) * (beta + 1)) * ((gamma + 1) * (delta + 1)) / (gamma + delta + 3)) * D[0];
    for (int i = 2; i < n; i++)
        D[i] = (2 * i + alpha + beta) / (2 * i + gamma + delta) * std::sqrt(((2 * i + alpha + beta - 1) * (2 * i + alpha + beta + 1)) / ((i + alpha) * (i + beta) * (i + alpha + beta)) * ((i + gamma) * (i + delta) * (i + gamma + delta)) / ((2 * i + gamma + delta - 1) * (2 * i + gamma + delta + 1))) * D[i - 1];
    return eigenvectors(A, B, D);
}

// ---------------------------------------------------------------------------
// Task lists of the rotation kernel.
// ---------------------------------------------------------------------------
double task_cost(int kind, int N, int M, int mbase) {
    const int step = Geo::step(kind);
    const int ord = Geo::task_orders(kind);
    const int mlast = Geo::last_order(kind, M);
    int omax = mbase + step * (ord - 1);
    if (omax > mlast) omax = mbase + step * ((mlast - mbase) / step);
    const int jlo = kind == TRI ? 0 : (mbase & 1);
    double cost = 0;
    for (int j = jlo; j <= omax - step; j += step) cost += std::max(0, Geo::top(kind, N, j, 0) + 2);
    return cost + 64.0;   // pipeline fill per pass, roughly
}

std::vector<RotTask> build_tasks(int kind, int N, int M, int field) {
    std::vector<RotTask> t;
    const int mfirst = Geo::first_order(kind), mlast = Geo::last_order(kind, M);
    const int span = Geo::step(kind) * Geo::task_orders(kind);
    if (kind == TRI) {
        for (int m = mfirst; m <= mlast; m += span) t.push_back({field, m});
    } else {
        for (int p = 0; p < 2; p++) {
            const int m0 = p == 0 ? 2 : 3;
            for (int m = m0; m <= mlast; m += span) t.push_back({field, m});
        }
    }
    return t;
}

}  // namespace ftb
