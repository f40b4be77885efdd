/*
 * CPU restatement of the BGK3D_HIT time-step hot path (TEST INFRASTRUCTURE).
 *
 * This file is the oracle: tests and the smoke check use it to check results,
 * the benchmark's CPU legs as the timed CPU baseline. Nothing in the product
 * library links, loads or calls it.
 *
 * Parity unpinned: the reference ships no tests, golden vectors or fixtures,
 * and its Fortran/MPI build cannot be compiled in this environment (no Fortran
 * compiler, no MPI). The restatement follows the reference sources line by
 * line; each function cites the file:line it restates (paths relative to the
 * reference project).
 *
 * This header is included once per storage form by bgk_oracle.c with:
 *   SUF        symbol suffix (_f64, _f32, _f16)
 *   STOR       storage type of a population value
 *   REAL       arithmetic type (mykind in SRC/precision.F90:19-38)
 *   SIN, COS, SQRT  REAL math functions
 *   ENC(L,x)   REAL deviation -> stored value
 *   DEC(L,s)   stored value -> REAL deviation
 *
 * Layout: 19 arrays with one ghost layer, Fortran order, i fastest, indices
 * 0..l+1 (SRC/alloca.F90:178-216). Population q (1-based in the reference) is
 * a[q-1]. b[18] exists but is never used (b19 is allocated and unused in the
 * reference, SRC/alloca.F90:216; pop 19 is updated in place in a19,
 * SRC/col_MC.F90:351).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define LAT CAT(orc_lat, SUF)
#define FN(name) CAT(name, SUF)

typedef struct {
    int l, m, n;
    long gx, gy, gz; /* ghosted extents */
    long ng;         /* ghosted cells */
    STOR *a[19];
    STOR *b[19];
    REAL scale, inv_scale;
    double les_cs; /* Smagorinsky constant cteS; 0 = BGK collision */
} LAT;

static inline long FN(gidx)(const LAT *L, long i, long j, long k) {
    return i + L->gx * (j + L->gy * k);
}

LAT *FN(orc_create)(int l, int m, int n) {
    LAT *L = (LAT *)calloc(1, sizeof(LAT));
    if (!L) return NULL;
    L->l = l; L->m = m; L->n = n;
    L->gx = l + 2; L->gy = m + 2; L->gz = n + 2;
    L->ng = L->gx * L->gy * L->gz;
    L->scale = (REAL)1; L->inv_scale = (REAL)1;
    for (int q = 0; q < 19; ++q) {
        /* calloc: a freshly allocated Fortran array on Linux reads as zeros
           (anonymous mmap), which is what the never-filled ghost layers of the
           second lattice hold in the reference. */
        L->a[q] = (STOR *)calloc((size_t)L->ng, sizeof(STOR));
        L->b[q] = (STOR *)calloc((size_t)L->ng, sizeof(STOR));
        if (!L->a[q] || !L->b[q]) return NULL;
    }
    return L;
}

void FN(orc_destroy)(LAT *L) {
    if (!L) return;
    for (int q = 0; q < 19; ++q) { free(L->a[q]); free(L->b[q]); }
    free(L);
}

/* Selects the LES collision of SRC/col_MC.F90:221-309 with cteS = cs
   (cs > 0) or the plain BGK collision (cs = 0). */
void FN(orc_set_les)(LAT *L, double cs) {
    L->les_cs = cs;
}

void FN(orc_set_scale)(LAT *L, double scale) {
    L->scale = (REAL)scale;
    L->inv_scale = (REAL)(1.0 / scale);
}

/* Equilibrium deviation of the initial condition, the exact arithmetic of
   SRC/init.F90:97-137 with cte1 = 0 (SRC/init.F90:65-69): the polynomial
   cxQQ = rf*(c.u) + qf*(3.0*(c.u)^2 - |u|^2), stored as crho*w*(cte1+cxQQ).
   The sign pattern of each linear term follows the reference text (e.g. cx10
   uses rf*(-xj-yj) and qf*(3*(xj+yj)^2 ...)). */
static void FN(eq_init_cell)(LAT *L, long g, REAL xj, REAL yj, REAL zj, REAL crho) {
    const REAL rf = (REAL)3.0, qf = (REAL)1.5, three = (REAL)3.0, zero = (REAL)0;
    const REAL p0 = (REAL)(1.0 / 3.0), p1 = (REAL)(1.0 / 18.0), p2 = (REAL)(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
    const REAL cte1 = zero;
    REAL cvsq = xj * xj + yj * yj + zj * zj;
    REAL cx[19];
    cx[0]  = rf * ( xj - yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
    cx[1]  = rf * ( xj - zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
    cx[2]  = rf * ( xj + yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
    cx[3]  = rf * ( xj + zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
    cx[4]  = rf * ( xj     ) + qf * (three * (xj     ) * (xj     ) - cvsq);
    cx[5]  = rf * (      zj) + qf * (three * (zj     ) * (zj     ) - cvsq);
    cx[6]  = rf * ( yj + zj) + qf * (three * (yj + zj) * (yj + zj) - cvsq);
    cx[7]  = rf * ( yj     ) + qf * (three * (yj     ) * (yj     ) - cvsq);
    cx[8]  = rf * ( yj - zj) + qf * (three * (yj - zj) * (yj - zj) - cvsq);
    cx[9]  = rf * (-xj - yj) + qf * (three * (xj + yj) * (xj + yj) - cvsq);
    cx[10] = rf * (-xj - zj) + qf * (three * (xj + zj) * (xj + zj) - cvsq);
    cx[11] = rf * (-xj + yj) + qf * (three * (xj - yj) * (xj - yj) - cvsq);
    cx[12] = rf * (-xj + zj) + qf * (three * (xj - zj) * (xj - zj) - cvsq);
    cx[13] = rf * (-xj     ) + qf * (three * (xj     ) * (xj     ) - cvsq);
    cx[14] = rf * (     -zj) + qf * (three * (zj     ) * (zj     ) - cvsq);
    cx[15] = rf * (-yj - zj) + qf * (three * (yj + zj) * (yj + zj) - cvsq);
    cx[16] = rf * (-yj     ) + qf * (three * (yj     ) * (yj     ) - cvsq);
    cx[17] = rf * (-yj + zj) + qf * (three * (yj - zj) * (yj - zj) - cvsq);
    cx[18] = rf * ((REAL)0.0) + qf * (three * ((REAL)0.0) * ((REAL)0.0) - cvsq);
    static const int wcls[19] = {2,2,2,2,1,1,2,1,2,2,2,2,2,1,1,2,1,2,0};
    for (int q = 0; q < 19; ++q) {
        REAL w = wcls[q] == 0 ? p0 : (wcls[q] == 1 ? p1 : p2);
        L->a[q][g] = ENC(L, crho * w * (cte1 + cx[q]));
    }
}

/* Taylor-Green initial condition, SRC/init.F90:83-141.
   faithful=1: coordinates in default (single) precision real()/0.5 literals
   and the single-precision literal pi (SRC/init.F90:42,84-88), and the
   pressure-consistent crho (SRC/init.F90:94-95).
   faithful=0: coordinates and pi in double precision and crho = 1 (the
   "rho = 1, populations at equilibrium" Taylor-Green configuration).
   Trigonometric functions come from the C library. Fills the full haloed box
   0..l+1 as the reference does. Offsets are zero (one rank). */
void FN(orc_init_tgv)(LAT *L, double u0d, int faithful) {
    const REAL u0 = (REAL)u0d;
    const REAL uno = (REAL)1;
    const int lx = L->l, ly = L->m, lz = L->n;
    /* pi as the reference stores it: a default-real literal (SRC/init.F90:42) */
    const REAL pi_f = (REAL)3.141592653589793238462643383279f;
    const REAL pi_d = (REAL)3.141592653589793238462643383279;
    const REAL pi = faithful ? pi_f : pi_d;
    for (long k = 0; k <= L->n + 1; ++k) {
        REAL z = faithful ? (REAL)(((float)k - 0.5f) / (float)lz)
                          : (REAL)(((double)k - 0.5) / (double)lz);
        for (long j = 0; j <= L->m + 1; ++j) {
            REAL y = faithful ? (REAL)(((float)j - 0.5f) / (float)ly)
                              : (REAL)(((double)j - 0.5) / (double)ly);
            for (long i = 0; i <= L->l + 1; ++i) {
                REAL x = faithful ? (REAL)(((float)i - 0.5f) / (float)lx)
                                  : (REAL)(((double)i - 0.5) / (double)lx);
                REAL xj = u0 * SIN((REAL)2 * pi * x) * COS((REAL)2 * pi * y) * COS((REAL)2 * pi * z);
                REAL yj = -(u0 * COS((REAL)2 * pi * x) * SIN((REAL)2 * pi * y) * COS((REAL)2 * pi * z));
                REAL zj = (REAL)0;
                REAL crho;
                if (faithful)
                    crho = uno + ((u0 * u0) / ((REAL)16.0 * (REAL)3.0)) *
                                 (COS((REAL)4 * pi * x) + COS((REAL)4 * pi * y)) * (COS((REAL)4 * pi * z) + (REAL)2);
                else
                    crho = uno;
                FN(eq_init_cell)(L, FN(gidx)(L, i, j, k), xj, yj, zj, crho);
            }
        }
    }
}

/* Equilibrium initial condition from a velocity field given on the interior
   (Fortran order, i fastest, l*m*n values per component) and a uniform
   density rho: the same per-cell arithmetic as SRC/init.F90:97-137 with crho
   replaced by rho. Ghost layers receive the periodic image. */
void FN(orc_init_velocity)(LAT *L, const double *u, const double *v, const double *w, double rho) {
    const long l = L->l, m = L->m, n = L->n;
    for (long k = 0; k <= n + 1; ++k)
        for (long j = 0; j <= m + 1; ++j)
            for (long i = 0; i <= l + 1; ++i) {
                long ii = (i + l - 1) % l, jj = (j + m - 1) % m, kk = (k + n - 1) % n;
                long s = ii + l * (jj + m * kk);
                FN(eq_init_cell)(L, FN(gidx)(L, i, j, k), (REAL)u[s], (REAL)v[s], (REAL)w[s], (REAL)rho);
            }
}

/* Periodic ghost fill of bcond_comm_step3 on one rank (every neighbour is the
   rank itself), SRC/bcond.comm.step3.F90:77-297: z+ (04,06,07,13,18 from
   plane n to plane 0), z- (02,09,11,15,16 from plane 1 to n+1), x+
   (01..05 from i=l to i=0), x- (10..14 from i=1 to l+1), y+ (03,07,08,09,12
   from j=m to j=0), y- (01,10,16,17,18 from j=1 to m+1). Each face plane spans
   the ghost rows of the other axes, in this order, so that edge ghosts receive
   their periodic image. */
void FN(orc_boundaries)(LAT *L) {
    const long l = L->l, m = L->m, n = L->n;
    static const int zp[5] = {4, 6, 7, 13, 18}, zm[5] = {2, 9, 11, 15, 16};
    static const int xp[5] = {1, 2, 3, 4, 5}, xm[5] = {10, 11, 12, 13, 14};
    static const int yp[5] = {3, 7, 8, 9, 12}, ym[5] = {1, 10, 16, 17, 18};
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[zp[p] - 1];
        for (long j = 0; j <= m + 1; ++j)
            for (long i = 0; i <= l + 1; ++i) A[FN(gidx)(L, i, j, 0)] = A[FN(gidx)(L, i, j, n)];
    }
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[zm[p] - 1];
        for (long j = 0; j <= m + 1; ++j)
            for (long i = 0; i <= l + 1; ++i) A[FN(gidx)(L, i, j, n + 1)] = A[FN(gidx)(L, i, j, 1)];
    }
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[xp[p] - 1];
        for (long k = 0; k <= n + 1; ++k)
            for (long j = 0; j <= m + 1; ++j) A[FN(gidx)(L, 0, j, k)] = A[FN(gidx)(L, l, j, k)];
    }
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[xm[p] - 1];
        for (long k = 0; k <= n + 1; ++k)
            for (long j = 0; j <= m + 1; ++j) A[FN(gidx)(L, l + 1, j, k)] = A[FN(gidx)(L, 1, j, k)];
    }
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[yp[p] - 1];
        for (long k = 0; k <= n + 1; ++k)
            for (long i = 0; i <= l + 1; ++i) A[FN(gidx)(L, i, 0, k)] = A[FN(gidx)(L, i, m, k)];
    }
    for (int p = 0; p < 5; ++p) {
        STOR *A = L->a[ym[p] - 1];
        for (long k = 0; k <= n + 1; ++k)
            for (long i = 0; i <= l + 1; ++i) A[FN(gidx)(L, i, m + 1, k)] = A[FN(gidx)(L, i, 1, k)];
    }
}

/* Source cell (i - cx, j - cy, k - cz) of each pull, SRC/col_MC.F90:113-131,
   with the D3Q19 velocity set of SRC/alloca.F90:57-175. */
static const int FN(CX)[19] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0};
static const int FN(CY)[19] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0};
static const int FN(CZ)[19] = {0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0};

/* Pulls the 19 populations of interior cell (i,j,k) (1-based interior
   indices). periodic=0 reads the ghost layers as they are; periodic=1 wraps
   the index modulo the box instead. */
static inline void FN(pull)(const LAT *L, STOR *const *A, long i, long j, long k, int periodic, REAL x[19]) {
    for (int q = 0; q < 19; ++q) {
        long si = i - FN(CX)[q], sj = j - FN(CY)[q], sk = k - FN(CZ)[q];
        if (periodic) {
            si = (si - 1 + L->l) % L->l + 1;
            sj = (sj - 1 + L->m) % L->m + 1;
            sk = (sk - 1 + L->n) % L->n + 1;
        }
        x[q] = DEC(L, A[q][FN(gidx)(L, si, sj, sk)]);
    }
}

/* Moments and BGK equilibrium deviation, SRC/col_MC.F90:133-219 (cte1 = 1,
   cte0 = 0, no forcing), in REAL arithmetic with the reference's evaluation
   order. Returns rho; fills e[19]. */
static inline REAL FN(equilibrium)(const REAL x[19], REAL e[19], REAL *ux, REAL *uy, REAL *uz) {
    const REAL uno = (REAL)1, cte1 = (REAL)1, cte0 = uno - cte1;
    const REAL rf = (REAL)3.0, qf = (REAL)1.5, tre = (REAL)3.0;
    const REAL p0 = (REAL)(1.0 / 3.0), p1 = (REAL)(1.0 / 18.0), p2 = (REAL)(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
    REAL rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
             + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
             + x[16] + x[17] + x[18] + cte1;
    REAL rhoinv = uno / rho;
    REAL vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
    REAL vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
    REAL vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
    *ux = vx; *uy = vy; *uz = vz;
    REAL vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
    REAL vsq = vx2 + vy2 + vz2;
    REAL vxpy = vx + vy; REAL qxpy = cte0 + qf * (tre * vxpy * vxpy - vsq);
    REAL vxmy = vx - vy; REAL qxmy = cte0 + qf * (tre * vxmy * vxmy - vsq);
    REAL vxpz = vx + vz; REAL qxpz = cte0 + qf * (tre * vxpz * vxpz - vsq);
    REAL vxmz = vx - vz; REAL qxmz = cte0 + qf * (tre * vxmz * vxmz - vsq);
    REAL vypz = vy + vz; REAL qypz = cte0 + qf * (tre * vypz * vypz - vsq);
    REAL vymz = vy - vz; REAL qymz = cte0 + qf * (tre * vymz * vymz - vsq);
    REAL qx = cte0 + qf * (tre * vx2 - vsq);
    REAL qy = cte0 + qf * (tre * vy2 - vsq);
    REAL qz = cte0 + qf * (tre * vz2 - vsq);
    REAL q0 = cte0 + qf * (-vsq);
    vx = rf * vx; vy = rf * vy; vz = rf * vz;
    vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
    vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;
    REAL rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
    e[0]  = rp2 * (+vxmy + qxmy) + cte1 * (rp2 - p2);
    e[1]  = rp2 * (+vxmz + qxmz) + cte1 * (rp2 - p2);
    e[2]  = rp2 * (+vxpy + qxpy) + cte1 * (rp2 - p2);
    e[3]  = rp2 * (+vxpz + qxpz) + cte1 * (rp2 - p2);
    e[4]  = rp1 * (+vx + qx) + cte1 * (rp1 - p1);
    e[5]  = rp1 * (+vz + qz) + cte1 * (rp1 - p1);
    e[6]  = rp2 * (+vypz + qypz) + cte1 * (rp2 - p2);
    e[7]  = rp1 * (+vy + qy) + cte1 * (rp1 - p1);
    e[8]  = rp2 * (+vymz + qymz) + cte1 * (rp2 - p2);
    e[9]  = rp2 * (-vxpy + qxpy) + cte1 * (rp2 - p2);
    e[10] = rp2 * (-vxpz + qxpz) + cte1 * (rp2 - p2);
    e[11] = rp2 * (-vxmy + qxmy) + cte1 * (rp2 - p2);
    e[12] = rp2 * (-vxmz + qxmz) + cte1 * (rp2 - p2);
    e[13] = rp1 * (-vx + qx) + cte1 * (rp1 - p1);
    e[14] = rp1 * (-vz + qz) + cte1 * (rp1 - p1);
    e[15] = rp2 * (-vypz + qypz) + cte1 * (rp2 - p2);
    e[16] = rp1 * (-vy + qy) + cte1 * (rp1 - p1);
    e[17] = rp2 * (-vymz + qymz) + cte1 * (rp2 - p2);
    e[18] = rp0 * (+q0) + cte1 * (rp0 - p0);
    return rho;
}

/* Collision frequency, SRC/hencol.F90:31, in REAL arithmetic. */
double FN(orc_omega)(double svisc) {
    REAL s = (REAL)svisc;
    REAL o = ((REAL)1 + (REAL)1) / (((REAL)6.0 * s) + (REAL)1.0);
    return (double)o;
}

#ifdef FAST16
/* Collision of the FP16 form (no reference counterpart: the reference stops
   on HALF_P, SRC/precision.F90:40-43). It works on the scaled stored values
   y = scale*(f - w) as floats, keeps dr = sum(f - w) apart from 1, treats each
   pair of opposite directions (q, opp q), q = 0..8, together and uses fused
   multiply-adds (C fmaf, correctly rounded):
     dr = sum(y)*inv, u = j(y)*(inv/(1 + dr)), a = -1.5|u|^2,
     kd = K*dr, kr = K + kd with K = omega*scale*w (per weight class),
     kr3 = 3*kr, kr45 = 4.5*kr, kra = fmaf(kr, a, kd),
     t = fmaf(kr45*cu, cu, kra),
     y'(q) = fmaf(kr3, cu, fmaf(1 - omega, y, t)),
     y'(opp q) = fmaf(-kr3, cu, fmaf(1 - omega, y, t)),
     y'(rest) = fmaf(1 - omega, y, kra)
   (the BGK update y' = (1 - omega) y + K dr + K(1 + dr)(+-3cu + 4.5cu^2 + a)
   regrouped).
   The sums are grouped as written; this is the definition the CUDA kernels
   follow operation for operation. */
static inline float FN(cdotu16)(int q, float ux, float uy, float uz) {
    const int cx = FN(CX)[q], cy = FN(CY)[q], cz = FN(CZ)[q];
    float cu = 0.0f;
    int first = 1;
    if (cx != 0) { cu = cx > 0 ? ux : -ux; first = 0; }
    if (cy != 0) { float t = cy > 0 ? uy : -uy; cu = first ? t : cu + t; first = 0; }
    if (cz != 0) { float t = cz > 0 ? uz : -uz; cu = first ? t : cu + t; }
    return cu;
}

static void FN(fast16_cell)(const float *y, float *out, float inv, float om1, const float kw[3]) {
    static const int opp[9] = {11, 12, 9, 10, 13, 14, 15, 16, 17};
    static const int wcls[19] = {2,2,2,2,1,1,2,1,2,2,2,2,2,1,1,2,1,2,0};
    const float sp = ((y[0] + y[1]) + (y[2] + y[3])) + y[4];
    const float sm = ((y[9] + y[10]) + (y[11] + y[12])) + y[13];
    const float s0 = (((y[5] + y[6]) + (y[7] + y[8])) + ((y[14] + y[15]) + (y[16] + y[17]))) + y[18];
    const float sum = (sp + sm) + s0;
    const float jx = sp - sm;
    const float jyp = ((y[2] + y[6]) + (y[7] + y[8])) + y[11];
    const float jym = ((y[0] + y[9]) + (y[15] + y[16])) + y[17];
    const float jzp = ((y[3] + y[5]) + (y[6] + y[12])) + y[17];
    const float jzm = ((y[1] + y[8]) + (y[10] + y[14])) + y[15];
    const float dr = sum * inv;
    const float r = inv / (1.0f + dr);
    const float ux = jx * r, uy = (jyp - jym) * r, uz = (jzp - jzm) * r;
    const float usq = fmaf(uz, uz, fmaf(uy, uy, ux * ux));
    const float a = -1.5f * usq;
    float kr3[3], kr45[3], kra[3];
    for (int c = 0; c < 3; ++c) {
        const float kd = kw[c] * dr, kr = kw[c] + kd;
        kr3[c] = 3.0f * kr;
        kr45[c] = 4.5f * kr;
        kra[c] = fmaf(kr, a, kd);
    }
    for (int q = 0; q < 9; ++q) {
        const int c = wcls[q], o = opp[q];
        const float cu = FN(cdotu16)(q, ux, uy, uz);
        const float t = fmaf(kr45[c] * cu, cu, kra[c]);
        out[q] = fmaf(kr3[c], cu, fmaf(om1, y[q], t));
        out[o] = fmaf(-kr3[c], cu, fmaf(om1, y[o], t));
    }
    out[18] = fmaf(om1, y[18], kra[0]);
}

/* The FP16 form with the Smagorinsky closure (the reference's LES block,
   SRC/col_MC.F90:221-309, on the FP16 form's moments). With the sums, dr, u
   and a of fast16_cell and rho = 1 + dr, Pi_neq comes from the second
   moments of the stored values minus the equilibrium's closed form
   (D3Q19: sum_q c_a c_b (f_eq - w)_q = dr delta_ab / 3 + rho u_a u_b):
     Mxx = sp + sm, Myy = jyp + jym, Mzz = jzp + jzm,
     Mxy = (y2 + y9) - (y0 + y11), Mxz = (y3 + y10) - (y1 + y12),
     Myz = (y6 + y15) - (y8 + y17),
     d3 = dr*(1/3), Paa = fmaf(Maa, inv, -fmaf(rho u_a, u_a, d3)),
     Pab = fmaf(Mab, inv, -(rho u_a * u_b))   (rho u_z formed for Pzz only),
     pt = Pxx^2 (+ fmaf chain of the others, off-diagonal ones doubled),
     tau = tauh + 0.5*sqrt(fmaf(cs18, sqrt(pt), tau2)), om = 1/tau;
   the relaxation is then fast16_cell's pair update with om in place of
   omega and K = (om*scale)*w per weight class formed per cell. */
static void FN(fast16_les_cell)(const float *y, float *out, float inv, float scale, float cs18, float tauh,
                                float tau2) {
    static const int opp[9] = {11, 12, 9, 10, 13, 14, 15, 16, 17};
    static const int wcls[19] = {2,2,2,2,1,1,2,1,2,2,2,2,2,1,1,2,1,2,0};
    const float wv[3] = {1.0f / 3.0f, 1.0f / 18.0f, 1.0f / 36.0f};
    const float sp = ((y[0] + y[1]) + (y[2] + y[3])) + y[4];
    const float sm = ((y[9] + y[10]) + (y[11] + y[12])) + y[13];
    const float s0 = (((y[5] + y[6]) + (y[7] + y[8])) + ((y[14] + y[15]) + (y[16] + y[17]))) + y[18];
    const float sum = (sp + sm) + s0;
    const float jx = sp - sm;
    const float jyp = ((y[2] + y[6]) + (y[7] + y[8])) + y[11];
    const float jym = ((y[0] + y[9]) + (y[15] + y[16])) + y[17];
    const float jzp = ((y[3] + y[5]) + (y[6] + y[12])) + y[17];
    const float jzm = ((y[1] + y[8]) + (y[10] + y[14])) + y[15];
    const float dr = sum * inv;
    const float r = inv / (1.0f + dr);
    const float ux = jx * r, uy = (jyp - jym) * r, uz = (jzp - jzm) * r;
    const float usq = fmaf(uz, uz, fmaf(uy, uy, ux * ux));
    const float a = -1.5f * usq;
    const float rho = 1.0f + dr;
    const float d3 = dr * (1.0f / 3.0f);
    const float rux = rho * ux, ruy = rho * uy;
    const float Pxx = fmaf(sp + sm, inv, -fmaf(rux, ux, d3));
    const float Pyy = fmaf(jyp + jym, inv, -fmaf(ruy, uy, d3));
    const float Pzz = fmaf(jzp + jzm, inv, -fmaf(rho * uz, uz, d3));
    const float Pxy = fmaf((y[2] + y[9]) - (y[0] + y[11]), inv, -(rux * uy));
    const float Pxz = fmaf((y[3] + y[10]) - (y[1] + y[12]), inv, -(rux * uz));
    const float Pyz = fmaf((y[6] + y[15]) - (y[8] + y[17]), inv, -(ruy * uz));
    float pt = Pxx * Pxx;
    pt = fmaf(Pyy, Pyy, pt);
    pt = fmaf(Pzz, Pzz, pt);
    pt = fmaf(2.0f * Pxy, Pxy, pt);
    pt = fmaf(2.0f * Pxz, Pxz, pt);
    pt = fmaf(2.0f * Pyz, Pyz, pt);
    const float tau = tauh + 0.5f * sqrtf(fmaf(cs18, sqrtf(pt), tau2));
    const float om = 1.0f / tau;
    const float om1 = 1.0f - om;
    const float oms = om * scale;
    float kr3[3], kr45[3], kra[3];
    for (int c = 0; c < 3; ++c) {
        const float K = oms * wv[c];
        const float kd = K * dr, kr = K + kd;
        kr3[c] = 3.0f * kr;
        kr45[c] = 4.5f * kr;
        kra[c] = fmaf(kr, a, kd);
    }
    for (int q = 0; q < 9; ++q) {
        const int c = wcls[q], o = opp[q];
        const float cu = FN(cdotu16)(q, ux, uy, uz);
        const float t = fmaf(kr45[c] * cu, cu, kra[c]);
        out[q] = fmaf(kr3[c], cu, fmaf(om1, y[q], t));
        out[o] = fmaf(-kr3[c], cu, fmaf(om1, y[o], t));
    }
    out[18] = fmaf(om1, y[18], kra[0]);
}
#endif

static inline REAL FN(ptotal)(const REAL x[19], const REAL e[19]);

/* One fused pull-stream + BGK collide over the interior followed by the swap
   of pops 01..18, SRC/col_MC.F90:98-421. omega is passed in REAL precision.
   periodic selects ghost reads (reference) or modulo indexing. */
void FN(orc_col_mc_omega)(LAT *L, double omegad, int periodic) {
    const REAL omega = (REAL)omegad;
    const long l = L->l, m = L->m, n = L->n;
    /* LES constants of SRC/col_MC.F90:305 in REAL arithmetic:
       18*(cteS)**2, 1/(2*omega1), (1/omega1)**2 */
    const int les = L->les_cs > 0.0;
    const REAL cs = (REAL)L->les_cs;
    const REAL cs18 = (REAL)18 * (cs * cs);
    const REAL tauh = (REAL)1 / ((REAL)2 * omega);
    const REAL tau2 = ((REAL)1 / omega) * ((REAL)1 / omega);
#ifdef FAST16
    const float inv = (float)L->inv_scale, om1 = 1.0f - (float)omega;
    const double wd[3] = {1.0 / 3.0, 1.0 / 18.0, 1.0 / 36.0};
    float kw[3];
    for (int c = 0; c < 3; ++c) kw[c] = (float)((double)(float)omega * (double)L->scale * wd[c]);
#endif
#pragma omp parallel for schedule(static)
    for (long k = 1; k <= n; ++k)
        for (long j = 1; j <= m; ++j)
            for (long i = 1; i <= l; ++i) {
                long g = FN(gidx)(L, i, j, k);
#ifdef FAST16
                float y[19], out[19];
                for (int q = 0; q < 19; ++q) {
                    long si = i - FN(CX)[q], sj = j - FN(CY)[q], sk = k - FN(CZ)[q];
                    if (periodic) {
                        si = (si - 1 + l) % l + 1;
                        sj = (sj - 1 + m) % m + 1;
                        sk = (sk - 1 + n) % n + 1;
                    }
                    y[q] = (float)L->a[q][FN(gidx)(L, si, sj, sk)];
                }
                if (les) FN(fast16_les_cell)(y, out, inv, (float)L->scale, cs18, tauh, tau2);
                else FN(fast16_cell)(y, out, inv, om1, kw);
                for (int q = 0; q < 18; ++q) L->b[q][g] = (STOR)out[q];
                L->a[18][g] = (STOR)out[18];
#else
                REAL x[19], e[19], ux, uy, uz;
                FN(pull)(L, L->a, i, j, k, periodic, x);
                (void)FN(equilibrium)(x, e, &ux, &uy, &uz);
                REAL om = omega;
                if (les) {
                    /* SRC/col_MC.F90:302-306 */
                    const REAL Ptotal = SQRT(FN(ptotal)(x, e));
                    const REAL Ts = tauh + SQRT(cs18 * Ptotal + tau2) / (REAL)2;
                    om = (REAL)1 / Ts;
                }
                for (int q = 0; q < 18; ++q) L->b[q][g] = ENC(L, x[q] - om * (x[q] - e[q]));
                L->a[18][g] = ENC(L, x[18] - om * (x[18] - e[18]));
#endif
            }
    for (int q = 0; q < 18; ++q) {
        STOR *c = L->a[q]; L->a[q] = L->b[q]; L->b[q] = c;
    }
}

void FN(orc_col_mc)(LAT *L, double svisc, int periodic) {
    FN(orc_col_mc_omega)(L, FN(orc_omega)(svisc), periodic);
}

/* One time step of the reference loop body without diagnostics:
   boundaries then col_MC (SRC/bgk3d_HIT.F90:131,140). */
void FN(orc_step)(LAT *L, double svisc) {
    FN(orc_boundaries)(L);
    FN(orc_col_mc)(L, svisc, 0);
}

#ifndef FAST16
/* The same step written for a CPU: per row, 19 source-row pointers into the
   ghosted arrays and a vectorisable loop over i (each lane performs exactly
   the operations of FN(equilibrium) and the relaxation, so the result is
   bit-identical to orc_step). Used as the timed CPU baseline. BGK collision
   only: with the LES collision selected it runs orc_step. */
void FN(orc_step_rows)(LAT *L, double svisc) {
    if (L->les_cs > 0.0) {
        FN(orc_step)(L, svisc);
        return;
    }
    FN(orc_boundaries)(L);
    const REAL omega = (REAL)FN(orc_omega)(svisc);
    const long l = L->l, m = L->m, n = L->n;
    const REAL uno = (REAL)1, cte1 = (REAL)1, cte0 = uno - cte1;
    const REAL rf = (REAL)3.0, qf = (REAL)1.5, tre = (REAL)3.0;
    const REAL p0 = (REAL)(1.0 / 3.0), p1 = (REAL)(1.0 / 18.0), p2 = (REAL)(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 1; k <= n; ++k)
        for (long j = 1; j <= m; ++j) {
            const STOR *restrict s[19];
            STOR *restrict d[19];
            for (int q = 0; q < 19; ++q) {
                s[q] = L->a[q] + FN(gidx)(L, 1 - FN(CX)[q], j - FN(CY)[q], k - FN(CZ)[q]);
                d[q] = (q < 18 ? L->b[q] : L->a[18]) + FN(gidx)(L, 1, j, k);
            }
#pragma omp simd
            for (long i = 0; i < l; ++i) {
                REAL x[19];
                for (int q = 0; q < 19; ++q) x[q] = s[q][i];
                REAL rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
                         + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
                         + x[16] + x[17] + x[18] + cte1;
                REAL rhoinv = uno / rho;
                REAL vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                REAL vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                REAL vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
                REAL vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
                REAL vsq = vx2 + vy2 + vz2;
                REAL vxpy = vx + vy; REAL qxpy = cte0 + qf * (tre * vxpy * vxpy - vsq);
                REAL vxmy = vx - vy; REAL qxmy = cte0 + qf * (tre * vxmy * vxmy - vsq);
                REAL vxpz = vx + vz; REAL qxpz = cte0 + qf * (tre * vxpz * vxpz - vsq);
                REAL vxmz = vx - vz; REAL qxmz = cte0 + qf * (tre * vxmz * vxmz - vsq);
                REAL vypz = vy + vz; REAL qypz = cte0 + qf * (tre * vypz * vypz - vsq);
                REAL vymz = vy - vz; REAL qymz = cte0 + qf * (tre * vymz * vymz - vsq);
                REAL qx = cte0 + qf * (tre * vx2 - vsq);
                REAL qy = cte0 + qf * (tre * vy2 - vsq);
                REAL qz = cte0 + qf * (tre * vz2 - vsq);
                REAL q0 = cte0 + qf * (-vsq);
                vx = rf * vx; vy = rf * vy; vz = rf * vz;
                vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
                vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;
                REAL rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
                REAL e[19];
                e[0]  = rp2 * (+vxmy + qxmy) + cte1 * (rp2 - p2);
                e[1]  = rp2 * (+vxmz + qxmz) + cte1 * (rp2 - p2);
                e[2]  = rp2 * (+vxpy + qxpy) + cte1 * (rp2 - p2);
                e[3]  = rp2 * (+vxpz + qxpz) + cte1 * (rp2 - p2);
                e[4]  = rp1 * (+vx + qx) + cte1 * (rp1 - p1);
                e[5]  = rp1 * (+vz + qz) + cte1 * (rp1 - p1);
                e[6]  = rp2 * (+vypz + qypz) + cte1 * (rp2 - p2);
                e[7]  = rp1 * (+vy + qy) + cte1 * (rp1 - p1);
                e[8]  = rp2 * (+vymz + qymz) + cte1 * (rp2 - p2);
                e[9]  = rp2 * (-vxpy + qxpy) + cte1 * (rp2 - p2);
                e[10] = rp2 * (-vxpz + qxpz) + cte1 * (rp2 - p2);
                e[11] = rp2 * (-vxmy + qxmy) + cte1 * (rp2 - p2);
                e[12] = rp2 * (-vxmz + qxmz) + cte1 * (rp2 - p2);
                e[13] = rp1 * (-vx + qx) + cte1 * (rp1 - p1);
                e[14] = rp1 * (-vz + qz) + cte1 * (rp1 - p1);
                e[15] = rp2 * (-vypz + qypz) + cte1 * (rp2 - p2);
                e[16] = rp1 * (-vy + qy) + cte1 * (rp1 - p1);
                e[17] = rp2 * (-vymz + qymz) + cte1 * (rp2 - p2);
                e[18] = rp0 * (+q0) + cte1 * (rp0 - p0);
                for (int q = 0; q < 19; ++q) d[q][i] = ENC(L, x[q] - omega * (x[q] - e[q]));
            }
        }
    for (int q = 0; q < 18; ++q) {
        STOR *c = L->a[q]; L->a[q] = L->b[q]; L->b[q] = c;
    }
}
#endif

/* Neumaier-compensated accumulation in double. */
typedef struct { double s, c; } FN(ksum);
static inline void FN(kadd)(FN(ksum) *a, double v) {
    double t = a->s + v;
    if (fabs(a->s) >= fabs(v)) a->c += (a->s - t) + v; else a->c += (v - t) + a->s;
    a->s = t;
}
static inline double FN(kval)(const FN(ksum) *a) { return a->s + a->c; }

/* Mean quantities from the local (un-pulled) populations, SRC/diagno.F90:73-130.
   out = {mean rho, mean ux, mean uy, mean uz, mean 0.5|u|^2}.
   faithful=1: sequential REAL sums in loop order, including the typo
   ztot = ytot + zj (SRC/diagno.F90:110), and the REAL normalisation of
   SRC/diagno.F90:117-121.
   faithful=0: per-cell REAL moments, compensated double sums, ztot summed. */
void FN(orc_diagno)(const LAT *L, int faithful, double out[5]) {
    const long l = L->l, m = L->m, n = L->n;
    const REAL uno = (REAL)1, cte1 = (REAL)1;
    REAL rtot = 0, xtot = 0, ytot = 0, ztot = 0, stot = 0;
    FN(ksum) kr = {0, 0}, kx = {0, 0}, ky = {0, 0}, kz = {0, 0}, ks = {0, 0};
    for (long k = 1; k <= n; ++k)
        for (long j = 1; j <= m; ++j)
            for (long i = 1; i <= l; ++i) {
                long g = FN(gidx)(L, i, j, k);
                REAL x[19];
                for (int q = 0; q < 19; ++q) x[q] = DEC(L, L->a[q][g]);
                REAL rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
                         + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
                         + x[16] + x[17] + x[18] + cte1;
                REAL rhoinv = uno / rho;
                REAL xj = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                REAL yj = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                REAL zj = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
                REAL ke = (REAL)0.5 * (xj * xj + yj * yj + zj * zj);
                if (faithful) {
                    rtot = rtot + rho;
                    xtot = xtot + xj;
                    ytot = ytot + yj;
                    ztot = ytot + zj;
                    stot = stot + ke;
                } else {
                    FN(kadd)(&kr, (double)rho); FN(kadd)(&kx, (double)xj);
                    FN(kadd)(&ky, (double)yj); FN(kadd)(&kz, (double)zj);
                    FN(kadd)(&ks, (double)ke);
                }
            }
    if (faithful) {
        REAL fl = (REAL)(float)l, fm = (REAL)(float)m, fn = (REAL)(float)n;
        out[0] = (double)((rtot / fl) / fm / fn);
        out[1] = (double)((xtot / fl) / fm / fn);
        out[2] = (double)((ytot / fl) / fm / fn);
        out[3] = (double)((ztot / fl) / fm / fn);
        out[4] = (double)((stot / fl) / fm / fn);
    } else {
        double vol = (double)l * (double)m * (double)n;
        out[0] = FN(kval)(&kr) / vol; out[1] = FN(kval)(&kx) / vol;
        out[2] = FN(kval)(&ky) / vol; out[3] = FN(kval)(&kz) / vol;
        out[4] = FN(kval)(&ks) / vol;
    }
}

/* Second moment of the non-equilibrium part, SRC/dissipation.F90:171-247:
   returns Ptotal = Pxx^2+Pyy^2+Pzz^2 + 2 Pxy^2 + 2 Pxz^2 + 2 Pyz^2. */
static inline REAL FN(ptotal)(const REAL x[19], const REAL e[19]) {
    REAL nn[18];
    for (int q = 0; q < 18; ++q) nn[q] = x[q] - e[q];
    REAL Pxx = nn[0] + nn[1] + nn[2] + nn[3] + nn[4] + nn[9] + nn[10] + nn[11] + nn[12] + nn[13];
    REAL Pyy = nn[0] + nn[2] + nn[6] + nn[7] + nn[8] + nn[9] + nn[11] + nn[15] + nn[16] + nn[17];
    REAL Pzz = nn[1] + nn[3] + nn[5] + nn[6] + nn[8] + nn[10] + nn[12] + nn[14] + nn[15] + nn[17];
    REAL Pxz = -nn[1] + nn[3] + nn[10] - nn[12];
    REAL Pxy = -nn[0] + nn[2] + nn[9] - nn[11];
    REAL Pyz = +nn[6] - nn[8] + nn[15] - nn[17];
    REAL Pyx = Pxy, Pzx = Pxz, Pzy = Pyz;
    return (Pxx * Pxx) + (Pyy * Pyy) + (Pzz * Pzz) + ((REAL)2.0 * Pxy * Pyx) + ((REAL)2.0 * Pxz * Pzx) + ((REAL)2.0 * Pyz * Pzy);
}

/* Dissipation and turbulent kinetic energy from the pulled populations,
   SRC/dissipation.F90:65-269. out = {itime*dt, tke/(l*m*n*u0^2), diss, tke}.
   faithful=1: the ghost layers are read as they are (stale, as in the
   reference, whose dissipation runs after the pointer swap), REAL sequential
   sums, and dx = (2.0*3.141592)/float(lx) in single precision
   (SRC/dissipation.F90:65-66).
   faithful=0: periodic pulls and compensated double sums (2*svisc*Ptotal and
   0.5*vsq are formed in REAL per cell, as in the reference, then summed in
   double).
   faithful=2: the stale ghost layers of faithful=1 with the compensated sums
   of faithful=0 (the CUDA path's faithful mode, whose sums are compensated
   in every mode). */
void FN(orc_dissipation)(const LAT *L, double sviscd, double u0d, int itime, int faithful, double out[4]) {
    const long l = L->l, m = L->m, n = L->n;
    const REAL svisc = (REAL)sviscd, u0 = (REAL)u0d;
    REAL dx = (REAL)((2.0f * 3.141592f) / (float)l);
    REAL dt = dx * u0;
    REAL diss = 0, tke = 0;
    FN(ksum) kd = {0, 0}, kt = {0, 0};
    for (long k = 1; k <= n; ++k)
        for (long j = 1; j <= m; ++j)
            for (long i = 1; i <= l; ++i) {
                REAL x[19], e[19], ux, uy, uz;
                FN(pull)(L, L->a, i, j, k, faithful == 0, x);
                (void)FN(equilibrium)(x, e, &ux, &uy, &uz);
                REAL vsq = ux * ux + uy * uy + uz * uz;
                REAL P = FN(ptotal)(x, e);
                if (faithful == 1) {
                    tke = tke + (REAL)0.5 * vsq;
                    diss = diss + (REAL)2.0 * svisc * P;
                } else {
                    FN(kadd)(&kt, (double)((REAL)0.5 * vsq));
                    FN(kadd)(&kd, (double)((REAL)2.0 * svisc * P));
                }
            }
    if (faithful == 1) {
        out[0] = (double)((REAL)(float)itime * dt);
        out[1] = (double)(tke / (REAL)(float)l / (REAL)(float)m / (REAL)(float)n / (u0 * u0));
        out[2] = (double)diss;
        out[3] = (double)tke;
    } else {
        double t = FN(kval)(&kt);
        out[0] = (double)((REAL)(float)itime * dt);
        out[1] = t / (double)l / (double)m / (double)n / ((double)u0 * (double)u0);
        out[2] = FN(kval)(&kd);
        out[3] = t;
    }
}

/* Diagnostics with no reference counterpart (compensated double sums):
   out[0] enstrophy = mean over cells of 0.5*|curl u|^2, u from the local
          moments, second-order central differences with periodic wrap;
   out[1] eps_strain = mean over cells of 2*nu*S:S with
          S = -3*omega*Pi_neq/(2*rho) from the pulled populations;
   out[2] number of cells whose local rho or u is not finite. */
void FN(orc_extras)(const LAT *L, double sviscd, double out[3]) {
    const long l = L->l, m = L->m, n = L->n;
    const long N = l * m * n;
    double *U = (double *)malloc(sizeof(double) * 3 * (size_t)N);
    const REAL uno = (REAL)1, cte1 = (REAL)1;
    long nonfinite = 0;
    for (long k = 1; k <= n; ++k)
        for (long j = 1; j <= m; ++j)
            for (long i = 1; i <= l; ++i) {
                long g = FN(gidx)(L, i, j, k);
                REAL x[19];
                for (int q = 0; q < 19; ++q) x[q] = DEC(L, L->a[q][g]);
                REAL rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
                         + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
                         + x[16] + x[17] + x[18] + cte1;
                REAL rhoinv = uno / rho;
                REAL xj = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
                REAL yj = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
                REAL zj = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
                long s = (i - 1) + l * ((j - 1) + m * (k - 1));
                U[s] = (double)xj; U[N + s] = (double)yj; U[2 * N + s] = (double)zj;
                if (!isfinite((double)rho) || !isfinite((double)xj) || !isfinite((double)yj) || !isfinite((double)zj))
                    ++nonfinite;
            }
    FN(ksum) ke = {0, 0}, ks = {0, 0};
    const double om = FN(orc_omega)(sviscd);
    for (long k = 0; k < n; ++k)
        for (long j = 0; j < m; ++j)
            for (long i = 0; i < l; ++i) {
                long ip = (i + 1) % l, im = (i + l - 1) % l;
                long jp = (j + 1) % m, jm = (j + m - 1) % m;
                long kp = (k + 1) % n, km = (k + n - 1) % n;
#define UU(c, a, b, d) U[(c) * N + (a) + l * ((b) + m * (d))]
                double dwdy = 0.5 * (UU(2, i, jp, k) - UU(2, i, jm, k));
                double dvdz = 0.5 * (UU(1, i, j, kp) - UU(1, i, j, km));
                double dudz = 0.5 * (UU(0, i, j, kp) - UU(0, i, j, km));
                double dwdx = 0.5 * (UU(2, ip, j, k) - UU(2, im, j, k));
                double dvdx = 0.5 * (UU(1, ip, j, k) - UU(1, im, j, k));
                double dudy = 0.5 * (UU(0, i, jp, k) - UU(0, i, jm, k));
#undef UU
                double wx = dwdy - dvdz, wy = dudz - dwdx, wz = dvdx - dudy;
                FN(kadd)(&ke, 0.5 * (wx * wx + wy * wy + wz * wz));
                REAL x[19], e[19], ux, uy, uz;
                FN(pull)(L, L->a, i + 1, j + 1, k + 1, 1, x);
                REAL rho = FN(equilibrium)(x, e, &ux, &uy, &uz);
                double P = (double)FN(ptotal)(x, e);
                double r = (double)rho;
                FN(kadd)(&ks, 2.0 * sviscd * (9.0 * om * om / (4.0 * r * r)) * P);
            }
    free(U);
    out[0] = FN(kval)(&ke) / (double)N;
    out[1] = FN(kval)(&ks) / (double)N;
    out[2] = (double)nonfinite;
}

/* Interior populations in stored form, q-major, Fortran order:
   out[q*l*m*n + (i-1) + l*((j-1) + m*(k-1))]. */
void FN(orc_get_pops)(const LAT *L, STOR *out) {
    const long l = L->l, m = L->m, n = L->n, N = l * m * n;
    for (int q = 0; q < 19; ++q)
        for (long k = 1; k <= n; ++k)
            for (long j = 1; j <= m; ++j)
                for (long i = 1; i <= l; ++i)
                    out[q * N + (i - 1) + l * ((j - 1) + m * (k - 1))] = L->a[q][FN(gidx)(L, i, j, k)];
}

/* Same as orc_get_pops, decoded to double deviations f - w. */
void FN(orc_get_dev)(const LAT *L, double *out) {
    const long l = L->l, m = L->m, n = L->n, N = l * m * n;
    for (int q = 0; q < 19; ++q)
        for (long k = 1; k <= n; ++k)
            for (long j = 1; j <= m; ++j)
                for (long i = 1; i <= l; ++i)
                    out[q * N + (i - 1) + l * ((j - 1) + m * (k - 1))] = (double)DEC(L, L->a[q][FN(gidx)(L, i, j, k)]);
}

void FN(orc_put_pops)(LAT *L, const STOR *in) {
    const long l = L->l, m = L->m, n = L->n, N = l * m * n;
    for (int q = 0; q < 19; ++q)
        for (long k = 1; k <= n; ++k)
            for (long j = 1; j <= m; ++j)
                for (long i = 1; i <= l; ++i)
                    L->a[q][FN(gidx)(L, i, j, k)] = in[q * N + (i - 1) + l * ((j - 1) + m * (k - 1))];
}

/* Ghost-layer access for the edge-ghost checks (SRC/boundaries.F90:68-97
   dumps the same edge values under CORNER_CHECK): value of population q
   (1-based) at ghosted index (i,j,k), 0..l+1. */
double FN(orc_ghost_value)(const LAT *L, int q, long i, long j, long k) {
    return (double)DEC(L, L->a[q - 1][FN(gidx)(L, i, j, k)]);
}

#undef LAT
#undef FN
