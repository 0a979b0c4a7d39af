/*
 * One- and two-electron integrals over contracted Cartesian Gaussian shells.
 *
 * TEST INFRASTRUCTURE ONLY (part of the oracle): it produces the molecular integrals
 * that pin the CPU oracle to the reference's end-to-end known answers
 * (test/input.aq:20-24, H2O/cc-pVDZ).  Role of src/integrals/{os,fmgamma,1eints,2eints}.cxx
 * in the reference; the method here is the McMurchie-Davidson Hermite expansion
 * (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978)), written from its published
 * recurrences:
 *   E^{i+1,j}_t = E^{i,j}_{t-1}/(2p) + X_PA E^{i,j}_t + (t+1) E^{i,j}_{t+1}
 *   E^{i,j+1}_t = E^{i,j}_{t-1}/(2p) + X_PB E^{i,j}_t + (t+1) E^{i,j}_{t+1}
 *   R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X_PQ R^{n+1}_{t,u,v}   (likewise u, v)
 *   R^n_{000} = (-2a)^n F_n(a |PQ|^2)
 * The Boys function F_n(T) uses its Taylor series with downward recursion for T < 35 and
 * the asymptotic F_0 with upward recursion beyond.
 *
 * Shell functions are monomials x^i y^j z^k (i+j+k = l) times the contracted radial part,
 * all components of a shell sharing the normalisation of x^l; the caller transforms to
 * pure harmonics.  Component order: for l, (i, j, k) with i descending, then j descending.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LMAX 4
#define NMAX (4 * LMAX + 1)

static double boys_series(int n, double T) {
    /* F_n(T) = exp(-T) sum_k (2T)^k / ((2n+1)(2n+3)...(2n+2k+1)) */
    double term = 1.0 / (2 * n + 1), sum = term;
    for (int k = 1; k < 400; k++) {
        term *= 2.0 * T / (2 * n + 2 * k + 1);
        sum += term;
        if (term < 1e-17 * sum) break;
    }
    return exp(-T) * sum;
}

static void boys(int nmax, double T, double* F) {
    if (T < 35.0) {
        F[nmax] = boys_series(nmax, T);
        const double e = exp(-T);
        for (int n = nmax - 1; n >= 0; n--) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
    } else {
        const double e = exp(-T);
        F[0] = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
        for (int n = 0; n < nmax; n++) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2.0 * T);
    }
}

/* E[i][j][t] for 1D, i <= la, j <= lb */
static void hermite_E(int la, int lb, double a, double b, double Ax, double Bx, double E[LMAX + 1][LMAX + 1][2 * LMAX + 1]) {
    const double p = a + b, mu = a * b / p, Px = (a * Ax + b * Bx) / p;
    const double XPA = Px - Ax, XPB = Px - Bx, XAB = Ax - Bx;
    memset(E, 0, sizeof(double) * (LMAX + 1) * (LMAX + 1) * (2 * LMAX + 1));
    E[0][0][0] = exp(-mu * XAB * XAB);
    for (int i = 0; i <= la; i++) {
        for (int j = 0; j <= lb; j++) {
            if (i == 0 && j == 0) continue;
            for (int t = 0; t <= i + j; t++) {
                double v;
                if (i > 0) {
                    v = XPA * E[i - 1][j][t];
                    if (t > 0) v += E[i - 1][j][t - 1] / (2 * p);
                    if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
                } else {
                    v = XPB * E[i][j - 1][t];
                    if (t > 0) v += E[i][j - 1][t - 1] / (2 * p);
                    if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
                }
                E[i][j][t] = v;
            }
        }
    }
}

/* R[t][u][v] = R^0_{tuv}(a, X,Y,Z) for t+u+v <= L */
static void hermite_R(int L, double a, double X, double Y, double Z, double* R /* [(L+1)^3] */) {
    double F[NMAX + 1];
    boys(L, a * (X * X + Y * Y + Z * Z), F);
    const int S = L + 1;
    /* Rn[n][t][u][v] built for decreasing n */
    double* Rn = (double*)calloc((size_t)(L + 1) * S * S * S, sizeof(double));
#define IDX(n, t, u, v) ((((size_t)(n) * S + (t)) * S + (u)) * S + (v))
    double f = 1.0;
    for (int n = 0; n <= L; n++) {
        Rn[IDX(n, 0, 0, 0)] = f * F[n];
        f *= -2.0 * a;
    }
    for (int tot = 1; tot <= L; tot++) {
        for (int n = 0; n + tot <= L; n++) {
            for (int t = 0; t <= tot; t++)
                for (int u = 0; u + t <= tot; u++) {
                    int v = tot - t - u;
                    double val;
                    if (t > 0) {
                        val = X * Rn[IDX(n + 1, t - 1, u, v)];
                        if (t > 1) val += (t - 1) * Rn[IDX(n + 1, t - 2, u, v)];
                    } else if (u > 0) {
                        val = Y * Rn[IDX(n + 1, t, u - 1, v)];
                        if (u > 1) val += (u - 1) * Rn[IDX(n + 1, t, u - 2, v)];
                    } else {
                        val = Z * Rn[IDX(n + 1, t, u, v - 1)];
                        if (v > 1) val += (v - 1) * Rn[IDX(n + 1, t, u, v - 2)];
                    }
                    Rn[IDX(n, t, u, v)] = val;
                }
        }
    }
    for (int t = 0; t <= L; t++)
        for (int u = 0; u <= L; u++)
            for (int v = 0; v <= L; v++) R[((size_t)t * S + u) * S + v] = (t + u + v <= L) ? Rn[IDX(0, t, u, v)] : 0.0;
#undef IDX
    free(Rn);
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_components(int l, int (*c)[3]) {
    int k = 0;
    for (int i = l; i >= 0; i--)
        for (int j = l - i; j >= 0; j--) {
            c[k][0] = i;
            c[k][1] = j;
            c[k][2] = l - i - j;
            k++;
        }
}

typedef struct {
    int l, nprim;
    double center[3];
    const double* exps;
    const double* coefs; /* already include primitive normalisation */
} Shell;

/* shells described by flat arrays; offsets computed here */
static void make_shells(int nsh, const int* l, const int* nprim, const double* centers, const double* exps,
                        const double* coefs, Shell* sh) {
    int off = 0;
    for (int s = 0; s < nsh; s++) {
        sh[s].l = l[s];
        sh[s].nprim = nprim[s];
        sh[s].center[0] = centers[3 * s];
        sh[s].center[1] = centers[3 * s + 1];
        sh[s].center[2] = centers[3 * s + 2];
        sh[s].exps = exps + off;
        sh[s].coefs = coefs + off;
        off += nprim[s];
    }
}

/* one-electron: S, T, V (nuclear attraction to charges Z at positions C) in Cartesian AOs */
int one_electron(int nsh, const int* l, const int* nprim, const double* centers, const double* exps,
                 const double* coefs, int natom, const double* Z, const double* Cnuc, double* S, double* T,
                 double* V) {
    Shell* sh = (Shell*)malloc(sizeof(Shell) * nsh);
    make_shells(nsh, l, nprim, centers, exps, coefs, sh);
    int* first = (int*)malloc(sizeof(int) * (nsh + 1));
    first[0] = 0;
    for (int s = 0; s < nsh; s++) first[s + 1] = first[s] + ncart(sh[s].l);
    const int n = first[nsh];
    memset(S, 0, sizeof(double) * n * n);
    memset(T, 0, sizeof(double) * n * n);
    memset(V, 0, sizeof(double) * n * n);
    int ca[15][3], cb[15][3];
    for (int A = 0; A < nsh; A++)
        for (int B = 0; B < nsh; B++) {
            const Shell* a = &sh[A];
            const Shell* b = &sh[B];
            cart_components(a->l, ca);
            cart_components(b->l, cb);
            for (int pa = 0; pa < a->nprim; pa++)
                for (int pb = 0; pb < b->nprim; pb++) {
                    const double al = a->exps[pa], be = b->exps[pb], p = al + be;
                    const double cc = a->coefs[pa] * b->coefs[pb];
                    double P[3];
                    for (int x = 0; x < 3; x++) P[x] = (al * a->center[x] + be * b->center[x]) / p;
                    /* Hermite coefficients with j up to l_b + 2 (the kinetic term needs them) */
                    double Eb[3][LMAX + 1][LMAX + 3][2 * LMAX + 5];
                    for (int x = 0; x < 3; x++) {
                        memset(Eb[x], 0, sizeof(Eb[x]));
                        const double XPA = P[x] - a->center[x], XPB = P[x] - b->center[x];
                        const double XAB = a->center[x] - b->center[x];
                        Eb[x][0][0][0] = exp(-al * be / p * XAB * XAB);
                        for (int i = 0; i <= a->l; i++)
                            for (int j = 0; j <= b->l + 2; j++) {
                                if (i == 0 && j == 0) continue;
                                for (int t = 0; t <= i + j; t++) {
                                    double v;
                                    if (i > 0) {
                                        v = XPA * Eb[x][i - 1][j][t];
                                        if (t > 0) v += Eb[x][i - 1][j][t - 1] / (2 * p);
                                        if (t + 1 <= i - 1 + j) v += (t + 1) * Eb[x][i - 1][j][t + 1];
                                    } else {
                                        v = XPB * Eb[x][i][j - 1][t];
                                        if (t > 0) v += Eb[x][i][j - 1][t - 1] / (2 * p);
                                        if (t + 1 <= i + j - 1) v += (t + 1) * Eb[x][i][j - 1][t + 1];
                                    }
                                    Eb[x][i][j][t] = v;
                                }
                            }
                    }
                    const double sp = sqrt(M_PI / p);
                    /* nuclear attraction Hermite integrals per nucleus */
                    const int L = a->l + b->l;
                    const int SR = L + 1;
                    double* Rs = (double*)malloc(sizeof(double) * SR * SR * SR * (natom > 0 ? natom : 1));
                    for (int c = 0; c < natom; c++)
                        hermite_R(L, p, P[0] - Cnuc[3 * c], P[1] - Cnuc[3 * c + 1], P[2] - Cnuc[3 * c + 2],
                                  Rs + (size_t)c * SR * SR * SR);
                    for (int ia = 0; ia < ncart(a->l); ia++)
                        for (int ib = 0; ib < ncart(b->l); ib++) {
                            const int* ea = ca[ia];
                            const int* eb = cb[ib];
                            double s1[3], t1[3];
                            for (int x = 0; x < 3; x++) {
                                const int i = ea[x], j = eb[x];
                                s1[x] = Eb[x][i][j][0] * sp;
                                /* 1D kinetic: -1/2 <i| d2/dx2 |j> */
                                double d2 = 4.0 * be * be * Eb[x][i][j + 2][0] * sp - 2.0 * be * (2 * j + 1) * s1[x];
                                if (j >= 2) d2 += j * (j - 1) * Eb[x][i][j - 2][0] * sp;
                                t1[x] = -0.5 * d2;
                            }
                            const double sv = s1[0] * s1[1] * s1[2];
                            const double tv = t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2];
                            double vv = 0.0;
                            for (int c = 0; c < natom; c++) {
                                const double* R = Rs + (size_t)c * SR * SR * SR;
                                double acc = 0.0;
                                for (int t = 0; t <= ea[0] + eb[0]; t++)
                                    for (int u = 0; u <= ea[1] + eb[1]; u++)
                                        for (int v = 0; v <= ea[2] + eb[2]; v++)
                                            acc += Eb[0][ea[0]][eb[0]][t] * Eb[1][ea[1]][eb[1]][u] *
                                                   Eb[2][ea[2]][eb[2]][v] * R[((size_t)t * SR + u) * SR + v];
                                vv -= Z[c] * 2.0 * M_PI / p * acc;
                            }
                            const int mu = first[A] + ia, nu = first[B] + ib;
                            S[mu * n + nu] += cc * sv;
                            T[mu * n + nu] += cc * tv;
                            V[mu * n + nu] += cc * vv;
                        }
                    free(Rs);
                }
        }
    free(first);
    free(sh);
    return n;
}

/* (mu nu | la si) over Cartesian AOs, full n^4 array, chemist's notation */
int two_electron(int nsh, const int* l, const int* nprim, const double* centers, const double* exps,
                 const double* coefs, double* eri) {
    Shell* sh = (Shell*)malloc(sizeof(Shell) * nsh);
    make_shells(nsh, l, nprim, centers, exps, coefs, sh);
    int* first = (int*)malloc(sizeof(int) * (nsh + 1));
    first[0] = 0;
    for (int s = 0; s < nsh; s++) first[s + 1] = first[s] + ncart(sh[s].l);
    const int n = first[nsh];
    const size_t n2 = (size_t)n * n, n3 = n2 * n;
    int ca[15][3], cb[15][3], cc[15][3], cd[15][3];
    static double Eab[3][LMAX + 1][LMAX + 1][2 * LMAX + 1], Ecd[3][LMAX + 1][LMAX + 1][2 * LMAX + 1];
    const int SR = 4 * LMAX + 1;
    double* R = (double*)malloc(sizeof(double) * SR * SR * SR);
    double* blk = (double*)malloc(sizeof(double) * 15 * 15 * 15 * 15);
    for (int A = 0; A < nsh; A++)
        for (int B = 0; B <= A; B++)
            for (int C = 0; C < nsh; C++)
                for (int D = 0; D <= C; D++) {
                    if (A * (A + 1) / 2 + B < C * (C + 1) / 2 + D) continue;
                    const Shell *a = &sh[A], *b = &sh[B], *c = &sh[C], *d = &sh[D];
                    const int na = ncart(a->l), nb = ncart(b->l), nc = ncart(c->l), nd = ncart(d->l);
                    cart_components(a->l, ca);
                    cart_components(b->l, cb);
                    cart_components(c->l, cc);
                    cart_components(d->l, cd);
                    memset(blk, 0, sizeof(double) * na * nb * nc * nd);
                    const int L = a->l + b->l + c->l + d->l;
                    const int S1 = L + 1;
                    for (int pa = 0; pa < a->nprim; pa++)
                        for (int pb = 0; pb < b->nprim; pb++) {
                            const double al = a->exps[pa], be = b->exps[pb], p = al + be;
                            const double cab = a->coefs[pa] * b->coefs[pb];
                            if (cab == 0.0) continue;
                            double P[3];
                            for (int x = 0; x < 3; x++) {
                                P[x] = (al * a->center[x] + be * b->center[x]) / p;
                                hermite_E(a->l, b->l, al, be, a->center[x], b->center[x], Eab[x]);
                            }
                            for (int pc = 0; pc < c->nprim; pc++)
                                for (int pd = 0; pd < d->nprim; pd++) {
                                    const double ga = c->exps[pc], de = d->exps[pd], q = ga + de;
                                    const double ccd = c->coefs[pc] * d->coefs[pd];
                                    if (ccd == 0.0) continue;
                                    double Q[3];
                                    for (int x = 0; x < 3; x++) {
                                        Q[x] = (ga * c->center[x] + de * d->center[x]) / q;
                                        hermite_E(c->l, d->l, ga, de, c->center[x], d->center[x], Ecd[x]);
                                    }
                                    const double alpha = p * q / (p + q);
                                    hermite_R(L, alpha, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], R);
                                    const double pref = cab * ccd * 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q));
                                    for (int ia = 0; ia < na; ia++)
                                        for (int ib = 0; ib < nb; ib++) {
                                            const int *ea = ca[ia], *eb = cb[ib];
                                            for (int ic = 0; ic < nc; ic++)
                                                for (int id = 0; id < nd; id++) {
                                                    const int *ec = cc[ic], *ed = cd[id];
                                                    double acc = 0.0;
                                                    for (int t = 0; t <= ea[0] + eb[0]; t++)
                                                        for (int u = 0; u <= ea[1] + eb[1]; u++)
                                                            for (int v = 0; v <= ea[2] + eb[2]; v++) {
                                                                const double e1 = Eab[0][ea[0]][eb[0]][t] *
                                                                                  Eab[1][ea[1]][eb[1]][u] *
                                                                                  Eab[2][ea[2]][eb[2]][v];
                                                                if (e1 == 0.0) continue;
                                                                double inner = 0.0;
                                                                for (int tt = 0; tt <= ec[0] + ed[0]; tt++)
                                                                    for (int uu = 0; uu <= ec[1] + ed[1]; uu++)
                                                                        for (int vv = 0; vv <= ec[2] + ed[2]; vv++) {
                                                                            const double e2 = Ecd[0][ec[0]][ed[0]][tt] *
                                                                                              Ecd[1][ec[1]][ed[1]][uu] *
                                                                                              Ecd[2][ec[2]][ed[2]][vv];
                                                                            const double sgn = ((tt + uu + vv) & 1) ? -1.0 : 1.0;
                                                                            inner += sgn * e2 *
                                                                                     R[((size_t)(t + tt) * S1 + (u + uu)) * S1 + (v + vv)];
                                                                        }
                                                                acc += e1 * inner;
                                                            }
                                                    blk[((ia * nb + ib) * nc + ic) * nd + id] += pref * acc;
                                                }
                                        }
                                }
                        }
                    /* scatter with the 8-fold permutational symmetry */
                    for (int ia = 0; ia < na; ia++)
                        for (int ib = 0; ib < nb; ib++)
                            for (int ic = 0; ic < nc; ic++)
                                for (int id = 0; id < nd; id++) {
                                    const double v = blk[((ia * nb + ib) * nc + ic) * nd + id];
                                    const size_t m = first[A] + ia, nn = first[B] + ib, k = first[C] + ic,
                                                 s = first[D] + id;
                                    eri[m * n3 + nn * n2 + k * n + s] = v;
                                    eri[nn * n3 + m * n2 + k * n + s] = v;
                                    eri[m * n3 + nn * n2 + s * n + k] = v;
                                    eri[nn * n3 + m * n2 + s * n + k] = v;
                                    eri[k * n3 + s * n2 + m * n + nn] = v;
                                    eri[s * n3 + k * n2 + m * n + nn] = v;
                                    eri[k * n3 + s * n2 + nn * n + m] = v;
                                    eri[s * n3 + k * n2 + nn * n + m] = v;
                                }
                }
    free(blk);
    free(R);
    free(first);
    free(sh);
    return n;
}
