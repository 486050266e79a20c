/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the label-indexed anisotropic
 * elastic FDTD step. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it; the product never does.
 *
 * This header is included twice by fdtd_oracle.c, once with REAL = float and
 * once with REAL = double, to stamp out oracle_forward_f32 / _f64.
 *
 * It restates, in plain C, the per-step arithmetic of the reference's
 * production label path (Jerome-Graves/pulse-echo-azimuthal-simulation):
 *   strains      sim/core/fdtd.py:1136-1164  (strains_zp, term order of :1141-1162)
 *   stress       sim/core/fdtd.py:594-689    (stress_lab_u: q moves :612-642,
 *                                             J-ascending rows :643-648,
 *                                             deferred damping :649-657)
 *   source       sim/core/fdtd.py:1798-1800
 *   velocity     sim/core/fdtd.py:1211-1244  (vel_zp: j-major x/y/z term order,
 *                                             arithmetic face density :1237-1240)
 *   record       sim/core/fdtd.py:1806-1813  (pressure / vx / vy / vz)
 * and the dense path's recording convention (sim/core/fdtd.py:909-918: stress
 * damped at the end of the step before the pressure is formed) when
 * p->damped_record is set.
 *
 * fma_mode selects how products are rounded:
 *   0  every multiply and add rounded separately (the reference's expressions
 *      evaluated literally; what gcc -ffp-contract=off gives for its kernels);
 *   1  a fused multiply-add exactly where the CUDA product kernels place one
 *      (strain taps, stress row accumulation, the dt*acc update and velocity
 *      taps), so that the product kernels are bit-exact against this oracle.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

/* a += b * c, rounded as the mode says */
static inline REAL FN(mac)(int fm, REAL a, REAL b, REAL c)
{
    if (fm) return FMA_FN(b, c, a);
    REAL t = b * c;
    return a + t;
}

/* Half-cell move of a strain field from its staggered position to another
 * (the product-set average of sim/core/fdtd.py:612-633): guards per moved
 * axis, taps summed z-major then y then x, then scaled by 1/4. */
static inline REAL FN(moved)(const REAL *g, long idx, int iz, int iy, int ix,
                             int nz, int ny, int nx, long sy, long sz,
                             int dz, int dy, int dx)
{
    int lz = 0, hz = 0, ly = 0, hy = 0, lx = 0, hx = 0;
    int ntap = 1;
    if (dz > 0) { if (iz > nz - 2) return 0; lz = 0; hz = 1; ntap *= 2; }
    else if (dz < 0) { if (iz < 1) return 0; lz = -1; hz = 0; ntap *= 2; }
    if (dy > 0) { if (iy > ny - 2) return 0; ly = 0; hy = 1; ntap *= 2; }
    else if (dy < 0) { if (iy < 1) return 0; ly = -1; hy = 0; ntap *= 2; }
    if (dx > 0) { if (ix > nx - 2) return 0; lx = 0; hx = 1; ntap *= 2; }
    else if (dx < 0) { if (ix < 1) return 0; lx = -1; hx = 0; ntap *= 2; }
    REAL acc = 0;
    int first = 1;
    for (int a0 = lz; a0 <= hz; ++a0)
        for (int a1 = ly; a1 <= hy; ++a1)
            for (int a2 = lx; a2 <= hx; ++a2) {
                REAL t = g[idx + a0 * sz + a1 * sy + a2];
                if (first) { acc = t; first = 0; }
                else acc = acc + t;
            }
    REAL w = (ntap == 4) ? (REAL)0.25 : ((ntap == 2) ? (REAL)0.5 : (REAL)1.0);
    return acc * w;
}

/* staggered position of each Voigt component: 0 = c, 1 = yz, 2 = xz, 3 = xy
 * (sim/core/fdtd.py:40-41, :606-607) */
static const int FN(VP)[6] = {0, 0, 0, 1, 2, 3};
static const int FN(POS)[4][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

int FN(oracle_forward)(const OracleProblem *p, REAL *traces, REAL *state_out)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx;
    const long sy = nx, sz = (long)nx * ny;
    const long ncell = (long)nz * ny * nx;
    const int nc = p->nc, fm = p->fma_mode;
    REAL c[4] = {0, 0, 0, 0};
    for (int j = 0; j < nc; ++j) c[j] = (REAL)p->coeffs[j];
    const REAL inv_h = (REAL)p->inv_h, dt = (REAL)p->dt, dt_h = (REAL)p->dt_h;
    const REAL *ctab = (const REAL *)p->ctab;   /* (n_mat, 36) */
    const REAL *rho = (const REAL *)p->rho;     /* (n_mat,) */
    const REAL *src_w = (const REAL *)p->src_w;
    const REAL *wav = (const REAL *)p->wavelet;
    const REAL *rec_w = (const REAL *)p->rec_w;
    const int32_t *mat = p->mats;
    const float *damp = p->damp;

    if (nc < 1 || nc > 4) return 1;
    for (long i = 0; i < ncell; ++i)
        if (mat[i] < 0 || mat[i] >= p->n_mat) return 2;

    REAL *buf = (REAL *)calloc((size_t)15 * ncell, sizeof(REAL));
    REAL *sval = (REAL *)malloc(sizeof(REAL) * (p->n_src > 0 ? p->n_src : 1) * 3);
    if (!buf || !sval) { free(buf); free(sval); return 3; }
    REAL *vx = buf, *vy = buf + ncell, *vz = buf + 2 * ncell;
    REAL *s[6], *g[6];
    for (int I = 0; I < 6; ++I) s[I] = buf + (3 + I) * ncell;
    for (int J = 0; J < 6; ++J) g[J] = buf + (9 + J) * ncell;

#ifdef _OPENMP
    if (p->n_threads > 0) omp_set_num_threads(p->n_threads);
#endif

    for (int n = 0; n < p->nt; ++n) {
        /* ---- strains from v (strains_zp, sim/core/fdtd.py:1139-1163) ---- */
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    long idx = iz * sz + iy * sy + ix;
                    REAL a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
                    for (int j = 0; j < nc; ++j) {
                        REAL cj = c[j];
                        if (ix >= j + 1 && ix < nx - j)
                            a1 = FN(mac)(fm, a1, cj, vx[idx + j] - vx[idx - (j + 1)]);
                        if (iy >= j + 1 && iy < ny - j)
                            a2 = FN(mac)(fm, a2, cj, vy[idx + j * sy] - vy[idx - (j + 1) * sy]);
                        if (iz >= j + 1 && iz < nz - j)
                            a3 = FN(mac)(fm, a3, cj, vz[idx + j * sz] - vz[idx - (j + 1) * sz]);
                        if (iy >= j && iy < ny - j - 1)
                            a4 = FN(mac)(fm, a4, cj, vz[idx + (j + 1) * sy] - vz[idx - j * sy]);
                        if (iz >= j && iz < nz - j - 1)
                            a4 = FN(mac)(fm, a4, cj, vy[idx + (j + 1) * sz] - vy[idx - j * sz]);
                        if (ix >= j && ix < nx - j - 1)
                            a5 = FN(mac)(fm, a5, cj, vz[idx + (j + 1)] - vz[idx - j]);
                        if (iz >= j && iz < nz - j - 1)
                            a5 = FN(mac)(fm, a5, cj, vx[idx + (j + 1) * sz] - vx[idx - j * sz]);
                        if (ix >= j && ix < nx - j - 1)
                            a6 = FN(mac)(fm, a6, cj, vy[idx + (j + 1)] - vy[idx - j]);
                        if (iy >= j && iy < ny - j - 1)
                            a6 = FN(mac)(fm, a6, cj, vx[idx + (j + 1) * sy] - vx[idx - j * sy]);
                    }
                    g[0][idx] = a1 * inv_h; g[1][idx] = a2 * inv_h; g[2][idx] = a3 * inv_h;
                    g[3][idx] = a4 * inv_h; g[4][idx] = a5 * inv_h; g[5][idx] = a6 * inv_h;
                }

        /* ---- stress with deferred damping (stress_lab_u, :643-657) ---- */
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    long idx = iz * sz + iy * sy + ix;
                    REAL q[4][6];
                    for (int pp = 0; pp < 4; ++pp)
                        for (int J = 0; J < 6; ++J) {
                            int sp = FN(VP)[J];
                            if (sp == pp) q[pp][J] = g[J][idx];
                            else q[pp][J] = FN(moved)(g[J], idx, iz, iy, ix, nz, ny, nx, sy, sz,
                                                      FN(POS)[pp][0] - FN(POS)[sp][0],
                                                      FN(POS)[pp][1] - FN(POS)[sp][1],
                                                      FN(POS)[pp][2] - FN(POS)[sp][2]);
                        }
                    const REAL *Cm = ctab + (long)mat[idx] * 36;
                    REAL dmp = damp ? (REAL)damp[idx] : (REAL)1;
                    for (int I = 0; I < 6; ++I) {
                        int pp = FN(VP)[I];
                        REAL acc = 0;
                        for (int J = 0; J < 6; ++J)
                            acc = FN(mac)(fm, acc, Cm[I * 6 + J], q[pp][J]);
                        REAL sv = s[I][idx] * dmp;
                        sv = FN(mac)(fm, sv, dt, acc);
                        s[I][idx] = sv;
                    }
                }

        /* ---- explosive source into s1..s3 (:1798-1800): gather all, then
         *      scatter in list order, so a repeated cell keeps its last entry ---- */
        {
            REAL wn = wav[n];
            for (int k = 0; k < p->n_src; ++k) {
                REAL add = wn * src_w[k];
                for (int I = 0; I < 3; ++I) sval[k * 3 + I] = s[I][p->src_idx[k]] + add;
            }
            for (int k = 0; k < p->n_src; ++k)
                for (int I = 0; I < 3; ++I) s[I][p->src_idx[k]] = sval[k * 3 + I];
        }

        /* ---- velocity (vel_zp, :1213-1244) ---- */
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    long idx = iz * sz + iy * sy + ix;
                    const REAL *s1 = s[0], *s2 = s[1], *s3 = s[2], *s4 = s[3], *s5 = s[4], *s6 = s[5];
                    REAL ax = 0, ay = 0, az = 0;
                    for (int j = 0; j < nc; ++j) {
                        REAL cj = c[j];
                        if (ix >= j && ix < nx - j - 1)
                            ax = FN(mac)(fm, ax, cj, s1[idx + (j + 1)] - s1[idx - j]);
                        if (ix >= j + 1 && ix < nx - j) {
                            ay = FN(mac)(fm, ay, cj, s6[idx + j] - s6[idx - (j + 1)]);
                            az = FN(mac)(fm, az, cj, s5[idx + j] - s5[idx - (j + 1)]);
                        }
                        if (iy >= j && iy < ny - j - 1)
                            ay = FN(mac)(fm, ay, cj, s2[idx + (j + 1) * sy] - s2[idx - j * sy]);
                        if (iy >= j + 1 && iy < ny - j) {
                            ax = FN(mac)(fm, ax, cj, s6[idx + j * sy] - s6[idx - (j + 1) * sy]);
                            az = FN(mac)(fm, az, cj, s4[idx + j * sy] - s4[idx - (j + 1) * sy]);
                        }
                        if (iz >= j && iz < nz - j - 1)
                            az = FN(mac)(fm, az, cj, s3[idx + (j + 1) * sz] - s3[idx - j * sz]);
                        if (iz >= j + 1 && iz < nz - j) {
                            ax = FN(mac)(fm, ax, cj, s5[idx + j * sz] - s5[idx - (j + 1) * sz]);
                            ay = FN(mac)(fm, ay, cj, s4[idx + j * sz] - s4[idx - (j + 1) * sz]);
                        }
                    }
                    REAL r0 = rho[mat[idx]];
                    REAL rvx = (ix < nx - 1) ? (REAL)0.5 * (r0 + rho[mat[idx + 1]]) : r0;
                    REAL rvy = (iy < ny - 1) ? (REAL)0.5 * (r0 + rho[mat[idx + sy]]) : r0;
                    REAL rvz = (iz < nz - 1) ? (REAL)0.5 * (r0 + rho[mat[idx + sz]]) : r0;
                    REAL dmp = damp ? (REAL)damp[idx] : (REAL)1;
                    REAL tx = dt_h * ax, ty = dt_h * ay, tz = dt_h * az;
                    tx = tx / rvx; ty = ty / rvy; tz = tz / rvz;
                    vx[idx] = (vx[idx] + tx) * dmp;
                    vy[idx] = (vy[idx] + ty) * dmp;
                    vz[idx] = (vz[idx] + tz) * dmp;
                }

        /* ---- receiver groups (:1806-1813): weighted sum in list order ---- */
        for (int r = 0; r < p->n_rec_groups; ++r) {
            REAL acc = 0;
            for (int64_t k = p->rec_off[r]; k < p->rec_off[r + 1]; ++k) {
                long q = (long)p->rec_idx[k];
                REAL val;
                if (p->record == 0) {
                    REAL a = s[0][q], b = s[1][q], cc = s[2][q];
                    if (p->damped_record && damp) {
                        REAL d = (REAL)damp[q];
                        a = a * d; b = b * d; cc = cc * d;
                    }
                    REAL t = a + b;
                    t = t + cc;
                    val = -t / (REAL)3.0;
                } else if (p->record == 1) val = vx[q];
                else if (p->record == 2) val = vy[q];
                else val = vz[q];
                REAL prod = val * rec_w[k];
                acc = acc + prod;
            }
            traces[(long)n * p->n_rec_groups + r] = acc;
        }
    }
    if (state_out) {
        memcpy(state_out, buf, sizeof(REAL) * 9 * ncell);
    }
    free(buf);
    free(sval);
    return 0;
}

#undef FN
#undef CAT
#undef CAT2
