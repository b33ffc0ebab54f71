/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle of the two-electron path.
 *
 * A plain-C restatement of the reference jax_qc FP64 algorithm, used by the
 * tests as the checker and by bench.py as the timed CPU baseline ("port").
 * The product (jax_examples_b200) never links, loads or calls this file.
 *
 * Every function follows the reference loop structure and arithmetic order
 * (file:line of the reference project given per function), so its results
 * match the reference to rounding.  Parity of this restatement against the
 * reference itself is pinned by tests/golden/ fixtures produced by running
 * the reference's own code (tests/golden/gen_golden.py).
 *
 * boys_mode selects the Boys function:
 *   0 = the reference's boys_fn as is (Taylor below t=0.01, upward recurrence
 *       from F_0 above; integrals/boys.py:34-109).  It loses accuracy for
 *       n>=3 at small t, which the reference then carries into its ERIs.
 *   1 = an accurate F_n (series e^-t sum (2t)^k/(2n+1)(2n+3)..(2n+2k+1) for
 *       t < 40, upward recurrence from the erf form above, long double).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXL 12

/* ---------------------------------------------------------------- Boys */

/* integrals/boys.py:34-48  (_f0_series) */
static double f0_series(double t) {
    return 1.0 - t / 3.0 + t * t / 10.0 - t * t * t / 42.0 + pow(t, 4) / 216.0 -
           pow(t, 5) / 1320.0 + pow(t, 6) / 9360.0 - pow(t, 7) / 75600.0;
}

/* integrals/boys.py:51-65  (_f0_erf / boys_f0) */
static double boys_f0_ref(double t) {
    if (t < 1e-2) return f0_series(t);
    return 0.5 * sqrt(M_PI / t) * erf(sqrt(t));
}

/* integrals/boys.py:68-83  (_fn_series) */
static double fn_series(int n, double t) {
    double result = 1.0 / (2 * n + 1), sign = -1.0, tp = t, fact = 1.0;
    for (int k = 1; k < 8; ++k) {
        fact *= k;
        result = result + sign * tp / (fact * (2 * n + 2 * k + 1));
        sign = -sign;
        tp = tp * t;
    }
    return result;
}

/* integrals/boys.py:86-109  (boys_fn) */
double oracle_boys_ref(int n, double t) {
    if (n == 0) return boys_f0_ref(t);
    double safe_t = t > 0 ? t : 1.0;
    double e = exp(-t);
    double fn = boys_f0_ref(t);
    for (int k = 0; k < n; ++k) {
        double next = ((2 * k + 1) * fn - e) / (2.0 * safe_t);
        fn = t > 0 ? next : 1.0 / (2.0 * (k + 1) + 1.0);
    }
    return t < 1e-2 ? fn_series(n, t) : fn;
}

/* Accurate F_n(t): convergent series below 40, upward recurrence above. */
double oracle_boys_exact(int n, double t) {
    if (t < 40.0) {
        long double lt = t, term = 1.0L / (2 * n + 1), sum = term;
        for (int k = 1; k < 400; ++k) {
            term *= 2.0L * lt / (2 * n + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-21L) break;
        }
        return (double)(expl(-lt) * sum);
    }
    long double lt = t, f = 0.5L * sqrtl(3.14159265358979323846264338327950288L / lt) * erfl(sqrtl(lt));
    long double e = expl(-lt);
    for (int k = 0; k < n; ++k) f = ((2 * k + 1) * f - e) / (2.0L * lt);
    return (double)f;
}

static double boys(int mode, int n, double t) {
    return mode == 0 ? oracle_boys_ref(n, t) : oracle_boys_exact(n, t);
}

void oracle_boys_array(int mode, const double *t, long long nt, int mmax, double *out) {
    #pragma omp parallel for schedule(static)
    for (long long i = 0; i < nt; ++i)
        for (int m = 0; m <= mmax; ++m) out[i * (mmax + 1) + m] = boys(mode, m, t[i]);
}

/* ------------------------------------------------------- MMD recurrences */

/* mcmurchie_davidson.py:39-50 : libint Cartesian order */
static int cart_comps(int l, int (*c)[3]) {
    int k = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
            c[k][0] = lx; c[k][1] = ly; c[k][2] = l - lx - ly; ++k;
        }
    return k;
}

/* mcmurchie_davidson.py:60-108 (hermite_e); E[i][j][t] with E[0][0][0]=1.
 * Output laid out as E[(i*(lb+1)+j)*(la+lb+1)+t]. */
void oracle_hermite_e(int la, int lb, double xpa, double xpb, double p, double *E) {
    int T = la + lb + 1;
#define EI(i, j, t) E[((i) * (lb + 1) + (j)) * T + (t)]
    memset(E, 0, sizeof(double) * (la + 1) * (lb + 1) * T);
    EI(0, 0, 0) = 1.0;
    double inv2p = 0.5 / p;
    for (int i = 0; i < la; ++i) {
        for (int t = 0; t <= i; ++t) {
            double tm1 = t - 1 >= 0 ? EI(i, 0, t - 1) : 0.0;
            double tt = EI(i, 0, t);
            double tp1 = t + 1 <= i + 1 ? EI(i, 0, t + 1) : 0.0;
            EI(i + 1, 0, t) = inv2p * tm1 + xpa * tt + (t + 1) * tp1;
        }
        EI(i + 1, 0, i + 1) = inv2p * EI(i, 0, i);
    }
    for (int j = 0; j < lb; ++j)
        for (int i = 0; i <= la; ++i) {
            for (int t = 0; t <= i + j; ++t) {
                double tm1 = t - 1 >= 0 ? EI(i, j, t - 1) : 0.0;
                double tt = EI(i, j, t);
                double tp1 = t + 1 <= i + j ? EI(i, j, t + 1) : 0.0;
                EI(i, j + 1, t) = inv2p * tm1 + xpb * tt + (t + 1) * tp1;
            }
            EI(i, j + 1, i + j + 1) = inv2p * EI(i, j, i + j);
        }
#undef EI
}

/* mcmurchie_davidson.py:113-172 (hermite_r_aux), n_max = 0 trimmed output.
 * R laid out as R[(t*(umax+1)+u)*(vmax+1)+v]. */
void oracle_hermite_r(int tmax, int umax, int vmax, double p, const double *PC, int mode, double *Rout) {
    int Lm = tmax + umax + vmax;
    int nt = tmax + 1, nu = umax + 1, nv = vmax + 1, nn = Lm + 1;
    double *R = (double *)calloc((size_t)nt * nu * nv * nn, sizeof(double));
#define RI(t, u, v, n) R[(((t) * nu + (u)) * nv + (v)) * nn + (n)]
    double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
    double m2p = -2.0 * p, pw = 1.0;
    for (int n = 0; n <= Lm; ++n) { RI(0, 0, 0, n) = pw * boys(mode, n, T); pw *= m2p; }
    double X = PC[0], Y = PC[1], Z = PC[2];
    for (int t = 0; t < tmax; ++t)
        for (int n = 0; n < Lm - t; ++n) {
            double rm1 = t - 1 >= 0 ? RI(t - 1, 0, 0, n + 1) : 0.0;
            RI(t + 1, 0, 0, n) = t * rm1 + X * RI(t, 0, 0, n + 1);
        }
    for (int u = 0; u < umax; ++u)
        for (int t = 0; t <= tmax; ++t)
            for (int n = 0; n < Lm - t - u; ++n) {
                double rm1 = u - 1 >= 0 ? RI(t, u - 1, 0, n + 1) : 0.0;
                RI(t, u + 1, 0, n) = u * rm1 + Y * RI(t, u, 0, n + 1);
            }
    for (int v = 0; v < vmax; ++v)
        for (int u = 0; u <= umax; ++u)
            for (int t = 0; t <= tmax; ++t)
                for (int n = 0; n < Lm - t - u - v; ++n) {
                    double rm1 = v - 1 >= 0 ? RI(t, u, v - 1, n + 1) : 0.0;
                    RI(t, u, v + 1, n) = v * rm1 + Z * RI(t, u, v, n + 1);
                }
    for (int t = 0; t < nt; ++t)
        for (int u = 0; u < nu; ++u)
            for (int v = 0; v < nv; ++v) Rout[(t * nu + u) * nv + v] = RI(t, u, v, 0);
#undef RI
    free(R);
}

/* obara_saika.py:227-332 (primitive_eri_block).  out[(i*ncb+j)*ncc*ncd + k*ncd + l]. */
void oracle_primitive_eri(double alpha, const double *A, int la, double beta, const double *B, int lb,
                          double gamma, const double *C, int lc, double delta, const double *D, int ld,
                          int mode, double *out) {
    double p = alpha + beta, q = gamma + delta, rho = p * q / (p + q);
    double P[3], Q[3], PQ[3];
    for (int x = 0; x < 3; ++x) {
        P[x] = (alpha * A[x] + beta * B[x]) / p;
        Q[x] = (gamma * C[x] + delta * D[x]) / q;
    }
    double ab2 = 0, cd2 = 0;
    for (int x = 0; x < 3; ++x) {
        ab2 += (A[x] - B[x]) * (A[x] - B[x]);
        cd2 += (C[x] - D[x]) * (C[x] - D[x]);
        PQ[x] = P[x] - Q[x];
    }
    double Kab = exp(-(alpha * beta / p) * ab2), Kcd = exp(-(gamma * delta / q) * cd2);
    int Tab = la + lb + 1, Tcd = lc + ld + 1;
    double Eab[3][(MAXL / 2 + 1) * (MAXL / 2 + 1) * (MAXL + 1)], Ecd[3][(MAXL / 2 + 1) * (MAXL / 2 + 1) * (MAXL + 1)];
    for (int x = 0; x < 3; ++x) {
        oracle_hermite_e(la, lb, P[x] - A[x], P[x] - B[x], p, Eab[x]);
        oracle_hermite_e(lc, ld, Q[x] - C[x], Q[x] - D[x], q, Ecd[x]);
    }
    int tm = la + lb + lc + ld;
    int n1 = tm + 1;
    double *R = (double *)malloc(sizeof(double) * n1 * n1 * n1);
    oracle_hermite_r(tm, tm, tm, rho, PQ, mode, R);
    double pref = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * Kab * Kcd;
    int ca[28][3], cb[28][3], cc[28][3], cd[28][3];
    int na = cart_comps(la, ca), nb = cart_comps(lb, cb), nc = cart_comps(lc, cc), nd = cart_comps(ld, cd);
#define EA(x, i, j, t) Eab[x][((i) * (lb + 1) + (j)) * Tab + (t)]
#define EC(x, i, j, t) Ecd[x][((i) * (ld + 1) + (j)) * Tcd + (t)]
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j)
            for (int k = 0; k < nc; ++k)
                for (int l = 0; l < nd; ++l) {
                    double acc = 0.0;
                    for (int t = 0; t <= ca[i][0] + cb[j][0]; ++t) {
                        double et = EA(0, ca[i][0], cb[j][0], t);
                        if (et == 0.0) continue;
                        for (int u = 0; u <= ca[i][1] + cb[j][1]; ++u) {
                            double eu = EA(1, ca[i][1], cb[j][1], u);
                            if (eu == 0.0) continue;
                            for (int v = 0; v <= ca[i][2] + cb[j][2]; ++v) {
                                double ev = EA(2, ca[i][2], cb[j][2], v);
                                if (ev == 0.0) continue;
                                for (int tp = 0; tp <= cc[k][0] + cd[l][0]; ++tp) {
                                    double ft = EC(0, cc[k][0], cd[l][0], tp);
                                    if (ft == 0.0) continue;
                                    double st = (tp & 1) ? -1.0 : 1.0;
                                    for (int up = 0; up <= cc[k][1] + cd[l][1]; ++up) {
                                        double fu = EC(1, cc[k][1], cd[l][1], up);
                                        if (fu == 0.0) continue;
                                        double stu = (up & 1) ? -st : st;
                                        for (int vp = 0; vp <= cc[k][2] + cd[l][2]; ++vp) {
                                            double fv = EC(2, cc[k][2], cd[l][2], vp);
                                            if (fv == 0.0) continue;
                                            double s = (vp & 1) ? -stu : stu;
                                            acc += s * et * eu * ev * ft * fu * fv *
                                                   R[((t + tp) * n1 + (u + up)) * n1 + (v + vp)];
                                        }
                                    }
                                }
                            }
                        }
                    }
                    out[((i * nb + j) * nc + k) * nd + l] = pref * acc;
                }
#undef EA
#undef EC
    free(R);
}

/* ------------------------------------------------------------ basis view */

typedef struct {
    int n_shell;
    const int *l, *nprim, *prim_off;
    const double *exps, *coefs, *centres; /* centres: 3 per shell */
} basis_t;

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

/* obara_saika.py:394-426 (contracted_eri_block) */
static void contracted_eri(const basis_t *b, int I, int J, int K, int L, int mode, double *block, double *tmp) {
    int la = b->l[I], lb = b->l[J], lc = b->l[K], ld = b->l[L];
    int n = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    for (int x = 0; x < n; ++x) block[x] = 0.0;
    for (int i = 0; i < b->nprim[I]; ++i)
        for (int j = 0; j < b->nprim[J]; ++j)
            for (int k = 0; k < b->nprim[K]; ++k)
                for (int m = 0; m < b->nprim[L]; ++m) {
                    int pi = b->prim_off[I] + i, pj = b->prim_off[J] + j, pk = b->prim_off[K] + k,
                        pm = b->prim_off[L] + m;
                    double w = b->coefs[pi] * b->coefs[pj] * b->coefs[pk] * b->coefs[pm];
                    oracle_primitive_eri(b->exps[pi], b->centres + 3 * I, la, b->exps[pj], b->centres + 3 * J, lb,
                                         b->exps[pk], b->centres + 3 * K, lc, b->exps[pm], b->centres + 3 * L, ld,
                                         mode, tmp);
                    for (int x = 0; x < n; ++x) block[x] += w * tmp[x];
                }
}

void oracle_contracted_eri(int n_shell, const int *l, const int *nprim, const int *prim_off, const double *exps,
                           const double *coefs, const double *centres, int I, int J, int K, int L, int mode,
                           double *block) {
    basis_t b = {n_shell, l, nprim, prim_off, exps, coefs, centres};
    double tmp[1296 * 16];
    contracted_eri(&b, I, J, K, L, mode, block, tmp);
}

/* eri.py:69-138: canonical shell quartets i>=j, k>=l, ij>=kl, 8-fold scatter
 * into the dense (n,n,n,n) tensor (Cartesian layout). */
void oracle_eri_tensor(int n_shell, const int *l, const int *nprim, const int *prim_off, const double *exps,
                       const double *coefs, const double *centres, int mode, int n, double *eri) {
    basis_t b = {n_shell, l, nprim, prim_off, exps, coefs, centres};
    int *off = (int *)malloc(sizeof(int) * (n_shell + 1));
    off[0] = 0;
    for (int s = 0; s < n_shell; ++s) off[s + 1] = off[s] + ncart(l[s]);
    long long npair = (long long)n_shell * (n_shell + 1) / 2;
    #pragma omp parallel
    {
        double *block = (double *)malloc(sizeof(double) * 1296 * 16);
        double *tmp = (double *)malloc(sizeof(double) * 1296 * 16);
        #pragma omp for schedule(dynamic, 1)
        for (long long ij = 0; ij < npair; ++ij) {
            int i = (int)((sqrt(8.0 * ij + 1) - 1) / 2);
            while ((long long)i * (i + 1) / 2 > ij) --i;
            while ((long long)(i + 1) * (i + 2) / 2 <= ij) ++i;
            int j = (int)(ij - (long long)i * (i + 1) / 2);
            for (int k = 0; k < n_shell; ++k)
                for (int ll = 0; ll <= k; ++ll) {
                    long long kl = (long long)k * (k + 1) / 2 + ll;
                    if (ij < kl) continue;
                    contracted_eri(&b, i, j, k, ll, mode, block, tmp);
                    int ni = ncart(l[i]), nj = ncart(l[j]), nk = ncart(l[k]), nl = ncart(l[ll]);
                    for (int a = 0; a < ni; ++a)
                        for (int bb = 0; bb < nj; ++bb)
                            for (int c = 0; c < nk; ++c)
                                for (int d = 0; d < nl; ++d) {
                                    double v = block[((a * nj + bb) * nk + c) * nl + d];
                                    long long m0 = off[i] + a, m1 = off[j] + bb, m2 = off[k] + c, m3 = off[ll] + d;
                                    long long N = n;
#define PUT(p, q, r, s) eri[(((p) * N + (q)) * N + (r)) * N + (s)] = v
                                    PUT(m0, m1, m2, m3); PUT(m1, m0, m2, m3); PUT(m0, m1, m3, m2); PUT(m1, m0, m3, m2);
                                    PUT(m2, m3, m0, m1); PUT(m2, m3, m1, m0); PUT(m3, m2, m0, m1); PUT(m3, m2, m1, m0);
#undef PUT
                                }
                }
        }
        free(block);
        free(tmp);
    }
    free(off);
}

/* screening.py:32-58: Q[i,j] = sqrt(max_ab (ab|ab)) over the diagonal of the block. */
void oracle_schwarz(int n_shell, const int *l, const int *nprim, const int *prim_off, const double *exps,
                    const double *coefs, const double *centres, int mode, double *Q) {
    basis_t b = {n_shell, l, nprim, prim_off, exps, coefs, centres};
    #pragma omp parallel
    {
        double *block = (double *)malloc(sizeof(double) * 1296 * 16);
        double *tmp = (double *)malloc(sizeof(double) * 1296 * 16);
        #pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < n_shell; ++i)
            for (int j = i; j < n_shell; ++j) {
                contracted_eri(&b, i, j, i, j, mode, block, tmp);
                int na = ncart(l[i]), nb = ncart(l[j]);
                double mx = 0.0;
                for (int a = 0; a < na; ++a)
                    for (int c = 0; c < nb; ++c) {
                        double v = block[((a * nb + c) * na + a) * nb + c];
                        if (v > mx) mx = v;
                    }
                Q[i * n_shell + j] = Q[j * n_shell + i] = sqrt(mx > 0 ? mx : 0.0);
            }
        free(block);
        free(tmp);
    }
}

/* fock.py:31-38: J_mn = sum_ls D_ls (mn|ls), K_mn = sum_ls D_ls (ms|ln). */
void oracle_jk_from_tensor(int n, const double *D, const double *eri, double *J, double *K) {
    long long N = n;
    #pragma omp parallel for schedule(static)
    for (long long m = 0; m < N; ++m)
        for (long long nn = 0; nn < N; ++nn) {
            double j = 0.0, k = 0.0;
            for (long long l = 0; l < N; ++l)
                for (long long s = 0; s < N; ++s) {
                    double d = D[l * N + s];
                    j += d * eri[((m * N + nn) * N + l) * N + s];
                    k += d * eri[((m * N + s) * N + l) * N + nn];
                }
            J[m * N + nn] = j;
            K[m * N + nn] = k;
        }
}

/* Direct J/K over an explicit list of canonical shell quartets, without the
 * dense tensor: each quartet's contracted block is digested into J/K with the
 * images of the 8-fold symmetry (duplicates weighted by 1/2 per coincidence),
 * so that sum over all canonical quartets equals fock.py:31-38 on the dense
 * tensor.  Used by the CPU baseline to time a bounded sample of a large
 * workload; the quartet list is (i, j, k, l) with i>=j, k>=l, ij>=kl. */
void oracle_jk_quartets(int n_shell, const int *l, const int *nprim, const int *prim_off, const double *exps,
                        const double *coefs, const double *centres, int mode, int n, long long n_quartets,
                        const int *quartets, const double *D, double *J, double *K) {
    basis_t b = {n_shell, l, nprim, prim_off, exps, coefs, centres};
    int *off = (int *)malloc(sizeof(int) * (n_shell + 1));
    off[0] = 0;
    for (int s = 0; s < n_shell; ++s) off[s + 1] = off[s] + ncart(l[s]);
    long long N = n;
    memset(J, 0, sizeof(double) * N * N);
    memset(K, 0, sizeof(double) * N * N);
    #pragma omp parallel
    {
        double *block = (double *)malloc(sizeof(double) * 1296 * 16);
        double *tmp = (double *)malloc(sizeof(double) * 1296 * 16);
        double *Jl = (double *)calloc(N * N, sizeof(double));
        double *Kl = (double *)calloc(N * N, sizeof(double));
        #pragma omp for schedule(dynamic, 16)
        for (long long q = 0; q < n_quartets; ++q) {
            int i = quartets[4 * q], j = quartets[4 * q + 1], k = quartets[4 * q + 2], ll = quartets[4 * q + 3];
            contracted_eri(&b, i, j, k, ll, mode, block, tmp);
            double s = 1.0;
            if (i == j) s *= 0.5;
            if (k == ll) s *= 0.5;
            if (i == k && j == ll) s *= 0.5;
            int ni = ncart(l[i]), nj = ncart(l[j]), nk = ncart(l[k]), nl = ncart(l[ll]);
            for (int a = 0; a < ni; ++a)
                for (int bb = 0; bb < nj; ++bb)
                    for (int c = 0; c < nk; ++c)
                        for (int d = 0; d < nl; ++d) {
                            double v = s * block[((a * nj + bb) * nk + c) * nl + d];
                            long long p0 = off[i] + a, p1 = off[j] + bb, p2 = off[k] + c, p3 = off[ll] + d;
                            /* J: A_pq accumulates 2v D_rs (both orientations of the ket) */
                            Jl[p0 * N + p1] += 2.0 * v * D[p2 * N + p3];
                            Jl[p2 * N + p3] += 2.0 * v * D[p0 * N + p1];
                            Kl[p0 * N + p3] += v * D[p2 * N + p1];
                            Kl[p1 * N + p3] += v * D[p2 * N + p0];
                            Kl[p0 * N + p2] += v * D[p3 * N + p1];
                            Kl[p1 * N + p2] += v * D[p3 * N + p0];
                        }
        }
        #pragma omp critical
        {
            for (long long x = 0; x < N * N; ++x) { J[x] += Jl[x]; K[x] += Kl[x]; }
        }
        free(block); free(tmp); free(Jl); free(Kl);
    }
    /* symmetrize: J = A + A^T, K = B + B^T */
    for (long long m = 0; m < N; ++m)
        for (long long nn = 0; nn <= m; ++nn) {
            double a = J[m * N + nn] + J[nn * N + m];
            J[m * N + nn] = J[nn * N + m] = a;
            double c = K[m * N + nn] + K[nn * N + m];
            K[m * N + nn] = K[nn * N + m] = c;
        }
    free(off);
}

/* ------------------------------------------------- one-electron matrices */

/* obara_saika.py:69-176: 1-D overlap sqrt(pi/p) E[i][j][0] up to (la+1, lb+1),
 * kinetic 1-D from shifted overlaps, products over x,y,z times K_AB. */
static void prim_st(double alpha, const double *A, int la, double beta, const double *B, int lb, double *S,
                    double *T) {
    double p = alpha + beta, P[3], ab2 = 0;
    for (int x = 0; x < 3; ++x) {
        P[x] = (alpha * A[x] + beta * B[x]) / p;
        ab2 += (A[x] - B[x]) * (A[x] - B[x]);
    }
    double K = exp(-(alpha * beta / p) * ab2);
    double S1[3][4][4], T1[3][4][4], E[5 * 5 * 9];
    int ne = la + lb + 3;
    for (int x = 0; x < 3; ++x) {
        oracle_hermite_e(la + 1, lb + 1, P[x] - A[x], P[x] - B[x], p, E);
        double sq = sqrt(M_PI / p);
        for (int i = 0; i <= la + 1; ++i)
            for (int j = 0; j <= lb + 1; ++j) S1[x][i][j] = sq * E[(i * (lb + 2) + j) * ne + 0];
        for (int i = 0; i <= la; ++i)
            for (int j = 0; j <= lb; ++j) {
                double t = 4.0 * alpha * beta * S1[x][i + 1][j + 1];
                if (i > 0 && j > 0) t += i * j * S1[x][i - 1][j - 1];
                if (j > 0) t -= 2.0 * alpha * j * S1[x][i + 1][j - 1];
                if (i > 0) t -= 2.0 * beta * i * S1[x][i - 1][j + 1];
                T1[x][i][j] = 0.5 * t;
            }
    }
    int ca[28][3], cb[28][3];
    int na = cart_comps(la, ca), nb = cart_comps(lb, cb);
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) {
            int ax = ca[i][0], ay = ca[i][1], az = ca[i][2], bx = cb[j][0], by = cb[j][1], bz = cb[j][2];
            S[i * nb + j] = K * S1[0][ax][bx] * S1[1][ay][by] * S1[2][az][bz];
            T[i * nb + j] = K * (T1[0][ax][bx] * S1[1][ay][by] * S1[2][az][bz] +
                                 S1[0][ax][bx] * T1[1][ay][by] * S1[2][az][bz] +
                                 S1[0][ax][bx] * S1[1][ay][by] * T1[2][az][bz]);
        }
}

/* obara_saika.py:179-222: -Z (2 pi/p) K_AB sum_tuv E E E R_tuv(p, P-C). */
static void prim_v(double alpha, const double *A, int la, double beta, const double *B, int lb, int natom,
                   const double *C, const double *Z, int mode, double *V) {
    double p = alpha + beta, P[3], ab2 = 0;
    for (int x = 0; x < 3; ++x) {
        P[x] = (alpha * A[x] + beta * B[x]) / p;
        ab2 += (A[x] - B[x]) * (A[x] - B[x]);
    }
    double K = exp(-(alpha * beta / p) * ab2);
    int Tn = la + lb + 1;
    double E[3][3 * 3 * 5];
    for (int x = 0; x < 3; ++x) oracle_hermite_e(la, lb, P[x] - A[x], P[x] - B[x], p, E[x]);
    int ca[28][3], cb[28][3];
    int na = cart_comps(la, ca), nb = cart_comps(lb, cb);
    int L = la + lb, n1 = L + 1;
    double R[9 * 9 * 9];
    for (int i = 0; i < na * nb; ++i) V[i] = 0.0;
    for (int c = 0; c < natom; ++c) {
        double PC[3] = {P[0] - C[3 * c], P[1] - C[3 * c + 1], P[2] - C[3 * c + 2]};
        oracle_hermite_r(L, L, L, p, PC, mode, R);
        double pref = -Z[c] * (2.0 * M_PI / p) * K;
        for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j) {
                double acc = 0.0;
                for (int t = 0; t <= ca[i][0] + cb[j][0]; ++t) {
                    double ex = E[0][(ca[i][0] * (lb + 1) + cb[j][0]) * Tn + t];
                    if (ex == 0.0) continue;
                    for (int u = 0; u <= ca[i][1] + cb[j][1]; ++u) {
                        double ey = E[1][(ca[i][1] * (lb + 1) + cb[j][1]) * Tn + u];
                        if (ey == 0.0) continue;
                        for (int v = 0; v <= ca[i][2] + cb[j][2]; ++v)
                            acc += ex * ey * E[2][(ca[i][2] * (lb + 1) + cb[j][2]) * Tn + v] * R[(t * n1 + u) * n1 + v];
                    }
                }
                V[i * nb + j] += pref * acc;
            }
    }
}

/* overlap.py:67-85, kinetic.py:42-59, nuclear.py:62-81 (Cartesian layout). */
void oracle_one_electron(int n_shell, const int *l, const int *nprim, const int *prim_off, const double *exps,
                         const double *coefs, const double *centres, int natom, const double *atom_xyz,
                         const double *charges, int mode, int n, double *S, double *T, double *V) {
    int *off = (int *)malloc(sizeof(int) * (n_shell + 1));
    off[0] = 0;
    for (int s = 0; s < n_shell; ++s) off[s + 1] = off[s] + ncart(l[s]);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n_shell; ++i)
        for (int j = i; j < n_shell; ++j) {
            double bs[36], bt[36], bv[36], ps[36], pt[36], pv[36];
            int na = ncart(l[i]), nb = ncart(l[j]);
            for (int x = 0; x < na * nb; ++x) bs[x] = bt[x] = bv[x] = 0.0;
            for (int a = 0; a < nprim[i]; ++a)
                for (int b = 0; b < nprim[j]; ++b) {
                    int pa = prim_off[i] + a, pb = prim_off[j] + b;
                    double w = coefs[pa] * coefs[pb];
                    prim_st(exps[pa], centres + 3 * i, l[i], exps[pb], centres + 3 * j, l[j], ps, pt);
                    prim_v(exps[pa], centres + 3 * i, l[i], exps[pb], centres + 3 * j, l[j], natom, atom_xyz,
                           charges, mode, pv);
                    for (int x = 0; x < na * nb; ++x) {
                        bs[x] += w * ps[x]; bt[x] += w * pt[x]; bv[x] += w * pv[x];
                    }
                }
            for (int a = 0; a < na; ++a)
                for (int b = 0; b < nb; ++b) {
                    long long r = off[i] + a, c = off[j] + b;
                    S[r * n + c] = S[c * n + r] = bs[a * nb + b];
                    T[r * n + c] = T[c * n + r] = bt[a * nb + b];
                    V[r * n + c] = V[c * n + r] = bv[a * nb + b];
                }
        }
    free(off);
}
