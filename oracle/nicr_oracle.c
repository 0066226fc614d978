/* Test infrastructure only (the oracle). Plain-C restatement of the reference
 * solver's explicit step and initialisation, used to check the CUDA path.
 * Parity is pinned: tests compare this code with the unmodified reference
 * (oracle/_ref, built from the reference sources) and with the committed golden
 * fixtures under tests/golden/.
 *
 * Citations: 2D = mpi2d/NiCr2D_grains.cpp, 3S = mpi3d-slab/NiCr3D_grains.cpp.
 * Every floating-point expression keeps the reference's operand order and
 * association (C evaluates left to right like C++; built with
 * -ffp-contract=off and no -march, as the reference's Makefiles build it).
 * Budgets use long double (x87 80-bit on x86-64), as the reference's do.
 * Arrays carry a one-cell ghost layer like the reference's Field (3S:158-170),
 * X slowest; ghost fill follows ghosts() (3S:173-191, 2D:154-169).
 */
#define _GNU_SOURCE
#include "nicr_oracle.h"
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

static const double PI_ = 3.14159265358979323846;
/* Physics (3S:73-79) */
#define PH_W 1e4
#define PH_KO 1e-9
#define PH_KC 7.5e-9
#define PH_KP 1.7e-10
#define PH_L 0.2
#define PH_BMO 2.21e-16
#define PH_BMC 3.5436e-20
#define PH_BOO 2.21e-18
#define PH_BOC 3.5436e-21
#define PH_CKO 2e-10
#define PH_CKCR 2e-10
#define PH_BULKO 0.
#define PH_LAYERCR 0.182
#define PH_OXO 0.56300203
#define PH_OXCR 0.35677915

enum { B_NUCO, B_NUCCR, B_CKO, B_CKCR, B_CLIPO, B_CLIPCR, B_BCO, B_BCCR, B_N };

struct omodel {
    nicr_config c;
    int dim, nx, ny, nz;
    size_t ntot;           /* ghosted element count                          */
    double *o, *cr, *p, *on, *crn, *pn, *muO, *muCr, *mo, *mc, *grain, *gb;
    double *eta_s2, *eta_pairs, *gb_initial;
    double **eta, **eta_new;
    int neta, has_eta, eta_dirty, grain_freed;
    double* seeds;         /* dim doubles per seed */
    long long* volumes;
    int nseeds;
    long double b[B_N];
    long long nuclei, clipped;
    long double initialO, initialCr;
    int center_seed_cells;
    double next_nucleation;
    long long steps_done;
    char err[1024];
};

/* ---------------------------------------------------------------- indexing */
static inline size_t IX(const omodel* m, int i, int j, int k) {
    if (m->dim == 2) return (size_t)i * (size_t)(m->ny + 2) + (size_t)j;
    return ((size_t)i * (size_t)(m->ny + 2) + (size_t)j) * (size_t)(m->nz + 2) + (size_t)k;
}
#define A(f, i, j, k) ((f)[IX(m, i, j, k)])
#define FOR_CELLS(m) for (int i = 1; i <= (m)->nx; ++i) for (int j = 1; j <= (m)->ny; ++j) \
    for (int k = ((m)->dim == 2 ? 0 : 1); k <= ((m)->dim == 2 ? 0 : (m)->nz); ++k)

static double* alloc_field(const omodel* m, double v) {
    double* a = (double*)malloc(m->ntot * sizeof(double));
    for (size_t q = 0; q < m->ntot; ++q) a[q] = v;
    return a;
}

/* std::min / std::max / std::clamp semantics (first argument wins ties) */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* ---------------------------------------------------------------- physics */
static double h_(double p) { return p * p * p * (10. - 15. * p + 6. * p * p); }           /* 3S:171 */
static double hp_(double p) { return 30. * p * p * (p - 1.) * (p - 1.); }                 /* 3S:87  */
static double min_image(double d, double period) { return d - period * round(d / period); } /* 3S:172 */
static double fmetal(double o, double cr) {                                               /* 3S:198-201 */
    return (6000000. * o * o + 583264.303945031 * cr * cr + 3200000. * o * cr
            - 298432. * o - 97045.64 * cr - 61732.2974223055);
}
static double foxide(double o, double cr) {                                               /* 3S:202-205 */
    return (12000000. * o * o + 7000000. * cr * cr - 13800000. * o * cr
            - 8880000. * o + 2680000. * cr + 1860990.);
}
static double mu_metal_o(double o, double cr) { return (12000000. * o + 3200000. * cr - 298432.); } /* 3S:206 */
static double mobility(const omodel* m, double conc, double p, double gb, int oxygen) {   /* 3S:207-215 */
    if (oxygen && !m->c.oxygen_diffusion) return 0.;
    double hh = h_(p), bm = oxygen ? PH_BMO : PH_BMC, bo = oxygen ? PH_BOO : PH_BOC;
    const double gbf = oxygen ? m->c.gb_factor_o : m->c.gb_factor_cr;
    const double active = m->c.grains ? gb : 0.;
    return conc * ((1. - hh) * bm * (1. + (gbf - 1.) * active) + hh * bo);
}
static double ref_gb_width(const nicr_config* c) {                                        /* 3S:88-90 */
    return c->gb_fwhm_grid * c->dx * sqrt(PI_) / (2. * sqrt(log(2.)));
}
static double eta_K(const nicr_config* c) {                                               /* 3S:91-95 */
    if (c->eta_kappa > 0.) return c->eta_kappa;
    const double ell = 3. * ref_gb_width(c) / 8.;
    return 2. * c->eta_W * ell * ell;
}
static double eta_ell(const nicr_config* c) { return sqrt(eta_K(c) / (2. * c->eta_W)); }  /* 3S:96 */
static double eta_A(const nicr_config* c) { return c->eta_oxide_penalty < 0. ? c->eta_W : c->eta_oxide_penalty; }
static double eta_scale(const nicr_config* c) { return ref_gb_width(c) / (8. * eta_ell(c) / 3.); } /* 3S:98-103 */
static double g_energy(double S, double P, double phi, const nicr_config* c) {            /* 3S:104-107 */
    const double H = h_(phi), d = S - (1. - H);
    return 0.25 * c->eta_W * d * d + c->eta_W * P + 0.5 * eta_A(c) * H * S;
}
static double g_deta(double e, double S, double phi, const nicr_config* c) {              /* 3S:108-110 */
    return e * (c->eta_W * (S - (1. - h_(phi)) + 2. * (S - e * e)) + eta_A(c) * h_(phi));
}
static double g_dphi(double S, double phi, const nicr_config* c) {                        /* 3S:111-113 */
    return 0.5 * hp_(phi) * (c->eta_W * (S - (1. - h_(phi))) + eta_A(c) * S);
}

/* ---------------------------------------------------------------- ghosts / lap */
static void ghosts(omodel* m, double* a) {                                                /* 3S:173-191 */
    if (m->dim == 2) {                                                                    /* 2D:154-169 */
        for (int j = 1; j <= m->ny; ++j) { A(a, 0, j, 0) = A(a, 1, j, 0); A(a, m->nx + 1, j, 0) = A(a, m->nx, j, 0); }
        for (int i = 0; i <= m->nx + 1; ++i) { A(a, i, 0, 0) = A(a, i, m->ny, 0); A(a, i, m->ny + 1, 0) = A(a, i, 1, 0); }
        return;
    }
    for (int j = 1; j <= m->ny; ++j) for (int k = 1; k <= m->nz; ++k) {
        A(a, 0, j, k) = A(a, 1, j, k); A(a, m->nx + 1, j, k) = A(a, m->nx, j, k);
    }
    for (int i = 0; i <= m->nx + 1; ++i) {
        for (int k = 1; k <= m->nz; ++k) { A(a, i, 0, k) = A(a, i, m->ny, k); A(a, i, m->ny + 1, k) = A(a, i, 1, k); }
        for (int j = 0; j <= m->ny + 1; ++j) { A(a, i, j, 0) = A(a, i, j, m->nz); A(a, i, j, m->nz + 1) = A(a, i, j, 1); }
    }
}
static double lap(const omodel* m, const double* a, int i, int j, int k) {               /* 3S:192-196, 2D:170-173 */
    const nicr_config* c = &m->c;
    if (m->dim == 2)
        return (A(a, i + 1, j, 0) - 2. * A(a, i, j, 0) + A(a, i - 1, j, 0)) / (c->dx * c->dx)
             + (A(a, i, j + 1, 0) - 2. * A(a, i, j, 0) + A(a, i, j - 1, 0)) / (c->dy * c->dy);
    return (A(a, i + 1, j, k) - 2. * A(a, i, j, k) + A(a, i - 1, j, k)) / (c->dx * c->dx)
         + (A(a, i, j + 1, k) - 2. * A(a, i, j, k) + A(a, i, j - 1, k)) / (c->dy * c->dy)
         + (A(a, i, j, k + 1) - 2. * A(a, i, j, k) + A(a, i, j, k - 1)) / (c->dz * c->dz);
}
static long double lsum(const omodel* m, const double* a) {                               /* 3S:389-392 */
    long double v = 0;
    FOR_CELLS(m) v += A(a, i, j, k);
    return v;
}

/* ---------------------------------------------------------------- RNG */
/* MT19937-64 (Matsumoto & Nishimura; the parameters of std::mt19937_64,
 * C++ [rand.predef]) and libstdc++'s uniform_real_distribution<double> over a
 * 64-bit engine: one draw, u = double(x) / 2^64, clamped below 1, then
 * u * (b - a) + a. Used at 3S:425-427, 2D:246-248. */
typedef struct { uint64_t mt[312]; int mti; } mt64;
static void mt_seed(mt64* r, uint64_t s) {
    r->mt[0] = s;
    for (int i = 1; i < 312; ++i) r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
    r->mti = 312;
}
static uint64_t mt_next(mt64* r) {
    static const uint64_t MAG[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    if (r->mti >= 312) {
        int i;
        for (i = 0; i < 312 - 156; ++i) {
            uint64_t x = (r->mt[i] & UM) | (r->mt[i + 1] & LM);
            r->mt[i] = r->mt[i + 156] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
        }
        for (; i < 311; ++i) {
            uint64_t x = (r->mt[i] & UM) | (r->mt[i + 1] & LM);
            r->mt[i] = r->mt[i + (156 - 312)] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
        }
        uint64_t x = (r->mt[311] & UM) | (r->mt[0] & LM);
        r->mt[311] = r->mt[155] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
        r->mti = 0;
    }
    uint64_t x = r->mt[r->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}
static double mt_uniform(mt64* r, double a, double b) {
    double u = (double)mt_next(r) / 18446744073709551616.0;
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    return u * (b - a) + a;
}

/* ---------------------------------------------------------------- Voronoi */
static double competitor_distance3(const omodel* m, int g, int owner, double x, double y, double z,
                                   double oY, double oZ, double rbest) {               /* 3S:395-406 */
    const double* s = m->seeds;
    double db = INFINITY;
    for (int im = -1; im <= 1; ++im) for (int jm = -1; jm <= 1; ++jm) {
        const double gy = s[3 * g + 1] + im * m->ny, gz = s[3 * g + 2] + jm * m->nz;
        const double ax = s[3 * g] - x, ay = gy - y, az = gz - z;
        const double rs = ax * ax + ay * ay + az * az;
        const double bx = s[3 * g] - s[3 * owner], by = gy - oY, bz = gz - oZ;
        const double sep = sqrt(bx * bx + by * by + bz * bz);
        if (sep > 1.e-14) db = smin(db, smax(0., (rs - rbest) / (2. * sep)));
    }
    return db;
}
static int voronoi(omodel* m) {                                                           /* 3S:407-467, 2D:233-291 */
    const nicr_config* c = &m->c;
    free(m->seeds); free(m->volumes);
    if (!c->grains) {
        m->nseeds = 1;
        m->seeds = (double*)calloc(3, sizeof(double));
        m->seeds[0] = 0.5 * c->nx; m->seeds[1] = 0.5 * c->ny; if (m->dim == 3) m->seeds[2] = 0.5 * c->nz;
        m->volumes = (long long*)calloc(1, sizeof(long long));
        m->volumes[0] = m->dim == 3 ? (long long)(c->nx * c->ny * c->nz) : (long long)(c->nx * c->ny);
        for (size_t q = 0; q < m->ntot; ++q) { m->grain[q] = 1.; m->gb[q] = 0.; }
        return 0;
    }
    int ng;
    if (m->dim == 3) {
        const double volume = (double)c->nx * c->ny * c->nz;
        const double ng_real = 6. * volume / (PI_ * pow(c->grain_diameter_grid, 3));
        if (!isfinite(ng_real) || ng_real > volume + .5) { snprintf(m->err, sizeof m->err, "Too many Voronoi sites for this grid."); return 1; }
        ng = (int)llround(ng_real); if (ng < 1) ng = 1;
        if (ng > volume) { snprintf(m->err, sizeof m->err, "Too many Voronoi sites for this grid."); return 1; }
        if (m->has_eta && ng > c->max_eta_fields) {
            snprintf(m->err, sizeof m->err, "3D grain count exceeds --max-eta-fields; increase grain diameter or check memory before increasing the limit.");
            return 1;
        }
    } else {
        const double area = (double)c->nx * c->ny;
        ng = (int)llround(4. * area / (PI_ * c->grain_diameter_grid * c->grain_diameter_grid)); if (ng < 1) ng = 1;
        if (ng > c->nx * c->ny) { snprintf(m->err, sizeof m->err, "Too many Voronoi sites for this grid."); return 1; }
    }
    const int D = m->dim;
    m->nseeds = ng;
    m->seeds = (double*)calloc((size_t)ng * 3, sizeof(double));
    m->volumes = (long long*)calloc((size_t)ng, sizeof(long long));
    double* s = m->seeds;
    mt64 rng; mt_seed(&rng, c->random_seed);
    for (int g = 0; g < ng; ++g) {
        s[D * g] = mt_uniform(&rng, 0., (double)c->nx);
        s[D * g + 1] = mt_uniform(&rng, 0., (double)c->ny);
        if (D == 3) s[D * g + 2] = mt_uniform(&rng, 0., (double)c->nz);
    }
    const int les = c->left_edge_sites;
    if (D == 3) {
        const int lim = ng < c->ny * c->nz ? ng : c->ny * c->nz;
        if (les < 0 || les > lim) { snprintf(m->err, sizeof m->err, "--left-face-sites must be between 0 and min(volume-based site count, ny*nz)."); return 1; }
        if (les > 0) {                                                                    /* 3S:430-449 */
            const int n = les;
            int rows = (int)llround(sqrt((double)n * c->ny / c->nz));
            const int rmax = n < c->ny ? n : c->ny;
            rows = rows < 1 ? 1 : (rows > rmax ? rmax : rows);
            if ((n + c->nz - 1) / c->nz > rows) rows = (n + c->nz - 1) / c->nz;
            int phY = (int)(mt_uniform(&rng, 0., 1.) * c->ny); if (phY > c->ny - 1) phY = c->ny - 1;
            int phZ = (int)(mt_uniform(&rng, 0., 1.) * c->nz); if (phZ > c->nz - 1) phZ = c->nz - 1;
            int g = 0;
            for (int r = 0; r < rows; ++r) {
                const int cols = n / rows + (r < n % rows ? 1 : 0);
                const int yy = (phY + (int)((long long)r * c->ny / rows)) % c->ny;
                for (int q = 0; q < cols; ++q) {
                    const int zz = (phZ + (int)((long long)q * c->nz / cols)) % c->nz;
                    s[3 * g] = 0.05 + 0.4 * mt_uniform(&rng, 0., 1.);
                    s[3 * g + 1] = yy + 0.5; s[3 * g + 2] = zz + 0.5; ++g;
                }
            }
            for (int q = n; q < ng; ++q) s[3 * q] = 1.5 + (c->nx - 1.5) * (s[3 * q] / c->nx);
        }
    } else {
        const int lim = ng < c->ny ? ng : c->ny;
        if (les < 0 || les > lim) { snprintf(m->err, sizeof m->err, "--left-edge-sites must be between 0 and min(area-based site count, ny)."); return 1; }
        if (les > 0) {                                                                    /* 2D:251-265 */
            int phase = (int)(mt_uniform(&rng, 0., 1.) * c->ny); if (phase > c->ny - 1) phase = c->ny - 1;
            for (int q = 0; q < les; ++q) {
                const int row = (phase + (int)(((long long)q * c->ny) / les)) % c->ny;
                s[2 * q] = 0.05 + 0.4 * mt_uniform(&rng, 0., 1.);
                s[2 * q + 1] = row + 0.5;
            }
            for (int q = les; q < ng; ++q) s[2 * q] = 1.5 + (c->nx - 1.5) * (s[2 * q] / c->nx);
        }
    }
    const double f2 = c->gb_fwhm_grid * c->gb_fwhm_grid;
    FOR_CELLS(m) {
        const double x = i - .5, y = j - .5, z = k - .5;
        int owner = 0; double rbest = INFINITY, oY = 0., oZ = 0.;
        for (int g = 0; g < ng; ++g) {
            if (D == 3) {
                const double yy = min_image(s[3 * g + 1] - y, c->ny), zz = min_image(s[3 * g + 2] - z, c->nz);
                const double ax = s[3 * g] - x;
                const double rr = ax * ax + yy * yy + zz * zz;
                if (rr < rbest) { rbest = rr; owner = g; oY = y + yy; oZ = z + zz; }
            } else {
                const double dy = min_image(s[2 * g + 1] - y, c->ny);
                const double r = (s[2 * g] - x) * (s[2 * g] - x) + dy * dy;
                if (r < rbest) { rbest = r; owner = g; oY = y + dy; }
            }
        }
        A(m->grain, i, j, k) = owner + 1; m->volumes[owner]++;
        double db = INFINITY;
        for (int g = 0; g < ng; ++g) {
            if (g == owner) continue;
            if (D == 3) db = smin(db, competitor_distance3(m, g, owner, x, y, z, oY, oZ, rbest));
            else for (int im = -1; im <= 1; ++im) {
                const double ym = s[2 * g + 1] + im * c->ny;
                const double rs = (s[2 * g] - x) * (s[2 * g] - x) + (ym - y) * (ym - y);
                const double sep = hypot(s[2 * g] - s[2 * owner], ym - oY);
                if (sep > 1.e-14) db = smin(db, smax(0., (rs - rbest) / (2. * sep)));
            }
        }
        A(m->gb, i, j, k) = ng == 1 ? 0. : exp(-4. * log(2.) * db * db / f2);
    }
    ghosts(m, m->grain); ghosts(m, m->gb);
    return 0;
}

/* ---------------------------------------------------------------- init */
static int center_oxide(omodel* m) {                                                      /* 3S:725-751, 2D:517-542 */
    const nicr_config* c = &m->c;
    const double x = 0.5 * ((double)c->nx + 1.), y = 0.5 * ((double)c->ny + 1.), z = 0.5 * ((double)c->nz + 1.);
    const double r = c->radius_grid;
    int mn = c->nx < c->ny ? c->nx : c->ny;
    if (m->dim == 3 && c->nz < mn) mn = c->nz;
    if (r >= 0.5 * ((double)mn - 1.)) {
        snprintf(m->err, sizeof m->err, m->dim == 3 ? "Center seed is too large: --radius-grid must be less than (min(nx,ny,nz)-1)/2."
                                                    : "Center seed is too large: --radius-grid must be less than (min(nx,ny)-1)/2.");
        return 1;
    }
    FOR_CELLS(m) {
        const double ddx = i - x, ddy = j - y, ddz = k - z;
        const double d2 = m->dim == 3 ? ddx * ddx + ddy * ddy + ddz * ddz : ddx * ddx + ddy * ddy;
        if (d2 <= r * r) {
            m->b[B_NUCO] += PH_OXO - A(m->o, i, j, k); m->b[B_NUCCR] += PH_OXCR - A(m->cr, i, j, k);
            A(m->o, i, j, k) = PH_OXO; A(m->cr, i, j, k) = PH_OXCR; A(m->p, i, j, k) = 1.;
            ++m->center_seed_cells;
        }
    }
    if (m->center_seed_cells == 0) { snprintf(m->err, sizeof m->err, "Center seed covers no cell centres: increase --radius-grid."); return 1; }
    ++m->nuclei;
    return 0;
}

static void init_eta(omodel* m) {                                                         /* 3S:469-494, 2D:293-327 */
    const nicr_config* c = &m->c;
    const int ng = m->nseeds, D = m->dim;
    const double* s = m->seeds;
    m->neta = ng;
    m->eta = (double**)calloc((size_t)ng, sizeof(double*));
    m->eta_new = (double**)calloc((size_t)ng, sizeof(double*));
    for (int g = 0; g < ng; ++g) { m->eta[g] = alloc_field(m, 0.); m->eta_new[g] = alloc_field(m, 0.); }
    const double ell = eta_ell(c) / c->dx;
    double* w = (double*)malloc((size_t)ng * sizeof(double));
    FOR_CELLS(m) {
        const int owner = (int)A(m->grain, i, j, k) - 1;
        const double x = i - .5, y = j - .5, z = k - .5;
        double norm = 0.;
        if (D == 3) {
            const double oy = y + min_image(s[3 * owner + 1] - y, c->ny), oz = z + min_image(s[3 * owner + 2] - z, c->nz);
            const double ax = s[3 * owner] - x, ay = oy - y, az = oz - z;
            const double rbest = ax * ax + ay * ay + az * az;
            for (int g = 0; g < ng; ++g) {
                w[g] = g == owner ? 1. : exp(-competitor_distance3(m, g, owner, x, y, z, oy, oz, rbest) / ell);
                norm += w[g];
            }
        } else {
            const double oy = y + min_image(s[2 * owner + 1] - y, c->ny);
            const double ax = s[2 * owner] - x, ay = oy - y;
            const double rbest = ax * ax + ay * ay;
            for (int g = 0; g < ng; ++g) {
                if (g == owner) { w[g] = 1.; norm += 1.; continue; }
                double dist = INFINITY;
                for (int im = -1; im <= 1; ++im) {
                    const double gy = s[2 * g + 1] + im * c->ny;
                    const double sep = hypot(s[2 * g] - s[2 * owner], gy - oy);
                    const double bx = s[2 * g] - x, by = gy - y;
                    const double r = bx * bx + by * by;
                    if (sep > 1.e-14) dist = smin(dist, smax(0., (r - rbest) / (2. * sep)));
                }
                w[g] = exp(-dist / ell); norm += w[g];
            }
        }
        const double metal = 1. - h_(A(m->p, i, j, k));
        for (int g = 0; g < ng; ++g) A(m->eta[g], i, j, k) = metal * w[g] / norm;
    }
    free(w);
}

static void rebuild_eta_mask(omodel* m) {                                                 /* 3S:495-507, 2D:328-340 */
    const double scale = eta_scale(&m->c);
    FOR_CELLS(m) {
        double S = 0., pairs = 0.;
        for (int g = 0; g < m->neta; ++g) { const double q = A(m->eta[g], i, j, k) * A(m->eta[g], i, j, k); pairs += S * q; S += q; }
        A(m->eta_s2, i, j, k) = S; A(m->eta_pairs, i, j, k) = pairs;
        A(m->gb, i, j, k) = scale * smin(1., 16. * pairs);
    }
    ghosts(m, m->gb);
}

void oracle_refresh(omodel* m) {                                                          /* 3S:597-620, 2D:412-434 */
    const nicr_config* c = &m->c;
    ghosts(m, m->o); ghosts(m, m->cr); ghosts(m, m->p);
    if (m->has_eta && (m->dim == 2 || c->eta_L > 0. || !c->frozen_eta_cache || m->eta_dirty)) {
        for (int g = 0; g < m->neta; ++g) ghosts(m, m->eta[g]);
        rebuild_eta_mask(m);
        m->eta_dirty = 0;
    }
    FOR_CELLS(m) {
        const double o = A(m->o, i, j, k), cr = A(m->cr, i, j, k);
        double hh = h_(A(m->p, i, j, k));
        A(m->muO, i, j, k) = (1. - hh) * mu_metal_o(o, cr) + hh * (24000000. * o - 13800000. * cr - 8880000.)
                           - 2. * PH_KO * lap(m, m->o, i, j, k);
        A(m->muCr, i, j, k) = (1. - hh) * (1166528.60789006 * cr + 3200000. * o - 97045.64)
                            + hh * (14000000. * cr - 13800000. * o + 2680000.)
                            - 2. * PH_KC * lap(m, m->cr, i, j, k);
    }
    ghosts(m, m->muO); ghosts(m, m->muCr);
    if (c->bc == NICR_BC_MU && c->oxygen_diffusion) {
        for (int j = 1; j <= m->ny; ++j)
            for (int k = (m->dim == 2 ? 0 : 1); k <= (m->dim == 2 ? 0 : m->nz); ++k)
                A(m->muO, 0, j, k) = 2. * c->mu_res - A(m->muO, 1, j, k);
    }
    for (size_t q = 0; q < m->ntot; ++q) {
        m->mo[q] = mobility(m, m->o[q], m->p[q], m->gb[q], 1);
        m->mc[q] = mobility(m, m->cr[q], m->p[q], m->gb[q], 0);
    }
}

void oracle_invalidate(omodel* m) { m->eta_dirty = 1; }

static void free_model(omodel* m) {
    double** fs[] = {&m->o, &m->cr, &m->p, &m->on, &m->crn, &m->pn, &m->muO, &m->muCr, &m->mo, &m->mc,
                     &m->grain, &m->gb, &m->eta_s2, &m->eta_pairs, &m->gb_initial};
    for (size_t q = 0; q < sizeof fs / sizeof fs[0]; ++q) { free(*fs[q]); *fs[q] = NULL; }
    for (int g = 0; g < m->neta; ++g) { free(m->eta[g]); free(m->eta_new[g]); }
    free(m->eta); free(m->eta_new); free(m->seeds); free(m->volumes);
}

omodel* oracle_create(const nicr_config* cfg, char* err, int errlen) {                    /* 3S:356-384, 2D:208-228 */
    omodel* m = (omodel*)calloc(1, sizeof(omodel));
    m->c = *cfg;
    const nicr_config* c = &m->c;
    m->dim = c->dim; m->nx = c->nx; m->ny = c->ny; m->nz = c->dim == 3 ? c->nz : 1;
    m->ntot = c->dim == 3 ? (size_t)(m->nx + 2) * (m->ny + 2) * (m->nz + 2) : (size_t)(m->nx + 2) * (m->ny + 2);
    m->has_eta = c->grain_evolution && c->grains;
    m->eta_dirty = 1;
    m->next_nucleation = c->nucleation_period;
    m->o = alloc_field(m, 0.); m->cr = alloc_field(m, 0.); m->p = alloc_field(m, 0.);
    m->on = alloc_field(m, 0.); m->crn = alloc_field(m, 0.); m->pn = alloc_field(m, 0.);
    m->muO = alloc_field(m, 0.); m->muCr = alloc_field(m, 0.); m->mo = alloc_field(m, 0.); m->mc = alloc_field(m, 0.);
    m->grain = alloc_field(m, 0.); m->gb = alloc_field(m, 0.);
    m->eta_s2 = alloc_field(m, 0.); m->eta_pairs = alloc_field(m, 0.);
    int rc = voronoi(m);
    if (!rc) {
        m->gb_initial = alloc_field(m, 0.);
        memcpy(m->gb_initial, m->gb, m->ntot * sizeof(double));
        FOR_CELLS(m) {
            A(m->o, i, j, k) = PH_BULKO; A(m->cr, i, j, k) = c->bulk_cr; A(m->p, i, j, k) = 0.;
            if (c->bc == NICR_BC_CONCENTRATION && i == 1) { A(m->o, i, j, k) = c->layer_o; A(m->cr, i, j, k) = PH_LAYERCR; }
        }
        m->initialO = lsum(m, m->o); m->initialCr = lsum(m, m->cr);
        if (c->nucleation == NICR_NUC_CENTER) rc = center_oxide(m);
    }
    if (!rc && m->has_eta) {
        if (m->nseeds > c->max_eta_fields) {
            snprintf(m->err, sizeof m->err, "Too many eta fields; check --max-eta-fields and memory.");
            rc = 1;
        } else {
            init_eta(m);
            if (m->dim == 3) m->grain_freed = 1;
        }
    }
    if (rc) {
        if (err) snprintf(err, (size_t)errlen, "%s", m->err);
        free_model(m); free(m);
        return NULL;
    }
    oracle_refresh(m);
    return m;
}

void oracle_destroy(omodel* m) { if (m) { free_model(m); free(m); } }
long long oracle_ncells(const omodel* m) { return (long long)m->nx * m->ny * m->nz; }
int oracle_neta(const omodel* m) { return m->neta; }
int oracle_nseeds(const omodel* m) { return m->nseeds; }
int oracle_center_seed_cells(const omodel* m) { return m->center_seed_cells; }
const char* oracle_error(const omodel* m) { return m->err; }

int oracle_get(omodel* m, const char* name, double* out) {
    const double* a = NULL;
    if (!strcmp(name, "o")) a = m->o; else if (!strcmp(name, "cr")) a = m->cr; else if (!strcmp(name, "p")) a = m->p;
    else if (!strcmp(name, "muO")) a = m->muO; else if (!strcmp(name, "muCr")) a = m->muCr;
    else if (!strcmp(name, "mo")) a = m->mo; else if (!strcmp(name, "mc")) a = m->mc;
    else if (!strcmp(name, "gb")) a = m->gb; else if (!strcmp(name, "grain")) a = m->grain_freed ? NULL : m->grain;
    else if (!strcmp(name, "eta_s2")) a = m->eta_s2; else if (!strcmp(name, "eta_pairs")) a = m->eta_pairs;
    else if (!strcmp(name, "gb_initial")) a = m->gb_initial;
    else if (!strncmp(name, "eta", 3)) { int g = atoi(name + 3) - 1; if (g >= 0 && g < m->neta) a = m->eta[g]; }
    if (!a) return 1;
    size_t q = 0;
    FOR_CELLS(m) out[q++] = A(a, i, j, k);
    return 0;
}

int oracle_set_fields(omodel* m, const double* o, const double* cr, const double* p, const double* eta) {
    size_t q = 0;
    const size_t n = (size_t)oracle_ncells(m);
    FOR_CELLS(m) {
        A(m->o, i, j, k) = o[q]; A(m->cr, i, j, k) = cr[q]; A(m->p, i, j, k) = p[q];
        if (eta) for (int g = 0; g < m->neta; ++g) A(m->eta[g], i, j, k) = eta[(size_t)g * n + q];
        ++q;
    }
    m->eta_dirty = 1;
    oracle_refresh(m);
    return 0;
}
void oracle_reset_inventory(omodel* m) { m->initialO = lsum(m, m->o); m->initialCr = lsum(m, m->cr); }

int oracle_scale_eta(omodel* m, int g, int i, int j, int k, double f) {
    if (g < 0 || g >= m->neta) return 1;
    if (m->dim == 2) k = 0;
    A(m->eta[g], i, j, k) *= f;
    m->eta_dirty = 1;
    return 0;
}

/* ---------------------------------------------------------------- step */
static double left_flux(const omodel* m, int j, int k) {                                  /* 3S:621-628, 2D:435-442 */
    const nicr_config* c = &m->c;
    if (c->bc != NICR_BC_MU || !c->oxygen_diffusion) return 0.;
    const double mf = mobility(m, c->surface_c_ref, A(m->p, 1, j, k), A(m->gb, 1, j, k), 1);
    return 2. * mf * (c->mu_res - A(m->muO, 1, j, k)) / c->dx;
}
static double div_flux(const omodel* m, const double* M, const double* mu, int i, int j, int k, int oxygen) { /* 3S:629-638 */
    const nicr_config* c = &m->c;
    const double right = -.5 * (A(M, i, j, k) + A(M, i + 1, j, k)) * (A(mu, i + 1, j, k) - A(mu, i, j, k)) / c->dx;
    double left = -.5 * (A(M, i - 1, j, k) + A(M, i, j, k)) * (A(mu, i, j, k) - A(mu, i - 1, j, k)) / c->dx;
    if (oxygen && i == 1 && c->bc == NICR_BC_MU) left = left_flux(m, j, k);
    const double top = -.5 * (A(M, i, j, k) + A(M, i, j + 1, k)) * (A(mu, i, j + 1, k) - A(mu, i, j, k)) / c->dy;
    const double bottom = -.5 * (A(M, i, j - 1, k) + A(M, i, j, k)) * (A(mu, i, j, k) - A(mu, i, j - 1, k)) / c->dy;
    if (m->dim == 2) return (left - right) / c->dx + (bottom - top) / c->dy;                /* 2D:443-450 */
    const double front = -.5 * (A(M, i, j, k) + A(M, i, j, k + 1)) * (A(mu, i, j, k + 1) - A(mu, i, j, k)) / c->dz;
    const double back = -.5 * (A(M, i, j, k - 1) + A(M, i, j, k)) * (A(mu, i, j, k) - A(mu, i, j, k - 1)) / c->dz;
    return (left - right) / c->dx + (bottom - top) / c->dy + (back - front) / c->dz;
}

static int eta_trial(omodel* m) {                                                         /* 3S:514-526, 2D:347-359 */
    const nicr_config* c = &m->c;
    const double K = eta_K(c);
    for (int g = 0; g < m->neta; ++g) FOR_CELLS(m) {
        const double force = g_deta(A(m->eta[g], i, j, k), A(m->eta_s2, i, j, k), A(m->p, i, j, k), c) - K * lap(m, m->eta[g], i, j, k);
        const double v = A(m->eta[g], i, j, k) - c->dt * c->eta_L * force;
        if (!isfinite(v) || v < -1.e-12 || v > 1. + 1.e-12) {
            if (m->dim == 3)
                snprintf(m->err, sizeof m->err, "Eta trial outside [0,1]: grain=%d cell=(%d,%d,%d) value=%.17g. All PDE fields rejected together; eta is never clipped. Check eta coefficients/dt.", g + 1, i, j, k, v);
            else
                snprintf(m->err, sizeof m->err, "Eta trial outside [0,1]: grain=%d cell=(%d,%d) value=%.17g. All PDE fields rejected together; eta is never clipped. Check eta coefficients/dt.", g + 1, i, j, v);
            return NICR_ERR_ETA_RANGE;
        }
        A(m->eta_new[g], i, j, k) = v;
    }
    return 0;
}

int oracle_step(omodel* m) {                                                              /* 3S:761-826, 2D:551-597 */
    const nicr_config* c = &m->c;
    long double before[B_N]; memcpy(before, m->b, sizeof before);
    const long long nb = m->nuclei, cb = m->clipped;
    const int D = m->dim;
    const int kk0 = D == 2 ? 0 : 1, kk1 = D == 2 ? 0 : m->nz;
    const size_t nface = (size_t)m->ny * (size_t)(kk1 - kk0 + 1);
    double* inlet = NULL;
    const int reset_inlet = c->bc == NICR_BC_CONCENTRATION && c->oxygen_diffusion;
    if (reset_inlet) {                                                                    /* enforce_legacy_layer 3S:593-596 */
        inlet = (double*)malloc(nface * sizeof(double));
        size_t q = 0;
        for (int j = 1; j <= m->ny; ++j) for (int k = kk0; k <= kk1; ++k) inlet[q++] = A(m->o, 1, j, k);
        for (int j = 1; j <= m->ny; ++j) for (int k = kk0; k <= kk1; ++k) {
            m->b[B_BCO] += c->layer_o - A(m->o, 1, j, k); A(m->o, 1, j, k) = c->layer_o;
        }
    }
    oracle_refresh(m);
    for (int j = 1; j <= m->ny; ++j) for (int k = kk0; k <= kk1; ++k) m->b[B_BCO] += c->dt * left_flux(m, j, k) / c->dx;
    int rc = 0;
    FOR_CELLS(m) {
        if (rc) break;
        const double oo = A(m->o, i, j, k), cc = A(m->cr, i, j, k), pp = A(m->p, i, j, k);
        double on = c->oxygen_diffusion ? oo + c->dt * div_flux(m, m->mo, m->muO, i, j, k, 1) : oo;
        double crn = cc + c->dt * div_flux(m, m->mc, m->muCr, i, j, k, 0);
        const double hp = 30. * pp * pp * (pp - 1.) * (pp - 1.);
        double fp = PH_W * (4. * pp * pp * pp - 6. * pp * pp + 2. * pp)
                  + hp * (foxide(oo, cc) - fmetal(oo, cc)) - 2. * PH_KP * lap(m, m->p, i, j, k);
        if (m->has_eta) fp += g_dphi(A(m->eta_s2, i, j, k), pp, c);
        double pn = pp - c->dt * PH_L * fp;
        if (c->ck == NICR_CK_LEGACY) {
            const double dO = -PH_CKO * ((PH_OXO - on) * h_(pn) - (PH_OXO - oo) * h_(pp)) / c->dt;
            const double dCr = -PH_CKCR * ((PH_OXCR - crn) * h_(pn) - (PH_OXCR - cc) * h_(pp)) / c->dt;
            on += dO; crn += dCr; m->b[B_CKO] += dO; m->b[B_CKCR] += dCr;
        }
        if (!isfinite(on) || !isfinite(crn) || !isfinite(pn)) {
            snprintf(m->err, sizeof m->err, "Nonfinite trial field: reduce dt / inspect the model; no update accepted.");
            rc = NICR_ERR_TRIAL_NONFINITE; break;
        }
        if (c->bounds == NICR_BOUNDS_LEGACY) {
            const double oc = sclamp(on, 0., 1.), ccr = sclamp(crn, 0., 1.);
            m->b[B_CLIPO] += oc - on; m->b[B_CLIPCR] += ccr - crn;
            if (oc != on || ccr != crn) ++m->clipped;
            on = oc; crn = ccr;
            if (pn > .99999) pn = 1.;
            if (pn < 1.e-5) pn = 0.;
        } else if (on < -1.e-12 || crn < -1.e-12 || on + crn > 1. + 1.e-12 || pn < -1.e-12 || pn > 1. + 1.e-12) {
            if (D == 3)
                snprintf(m->err, sizeof m->err, "Out-of-bounds trial at (%d,%d,%d): O=%.16e, Cr=%.16e, phi=%.16e. No clipping/update accepted. Reduce dt; if failure persists, investigate model.", i, j, k, on, crn, pn);
            else
                snprintf(m->err, sizeof m->err, "Out-of-bounds trial at (%d,%d): O=%.16e, Cr=%.16e, phi=%.16e. No clipping/update accepted. Reduce dt; if failure persists, investigate model.", i, j, on, crn, pn);
            rc = NICR_ERR_TRIAL_BOUNDS; break;
        }
        A(m->on, i, j, k) = on; A(m->crn, i, j, k) = crn; A(m->pn, i, j, k) = pn;
    }
    const int advance_eta = m->has_eta && (D == 2 || c->eta_L > 0.);
    if (!rc && advance_eta) rc = eta_trial(m);
    if (rc) {
        /* Rejected: the budget rolls back (3S:812-820 and run() 2D:1224-1225); the
         * 3D inlet column is restored, the 2D one keeps the enforced layer. */
        memcpy(m->b, before, sizeof before); m->nuclei = nb; m->clipped = cb;
        if (reset_inlet && D == 3) {
            size_t q = 0;
            for (int j = 1; j <= m->ny; ++j) for (int k = kk0; k <= kk1; ++k) A(m->o, 1, j, k) = inlet[q++];
        }
        free(inlet);
        return rc;
    }
    free(inlet);
    double* t;
    t = m->o; m->o = m->on; m->on = t;
    t = m->cr; m->cr = m->crn; m->crn = t;
    t = m->p; m->p = m->pn; m->pn = t;
    if (advance_eta) {
        for (int g = 0; g < m->neta; ++g) { t = m->eta[g]; m->eta[g] = m->eta_new[g]; m->eta_new[g] = t; }
        m->eta_dirty = 1;
    }
    ++m->steps_done;
    return 0;
}

/* ---------------------------------------------------------------- nucleation */
typedef struct { int count; int lo[2], hi[2]; } axis_nb;
static int bounded_reach(double radius, int n) { return radius >= n ? n : (int)ceil(radius); }   /* 3S:220 */
static axis_nb periodic_nb(int center, double radius, int n) {                                     /* 3S:221-231 */
    const int r = bounded_reach(radius, n);
    axis_nb a; memset(&a, 0, sizeof a);
    if (2LL * r + 1 >= n) { a.count = 1; a.lo[0] = 1; a.hi[0] = n; return a; }
    const long long lo = (long long)center - r, hi = (long long)center + r;
    if (lo < 1) { a.count = 2; a.lo[0] = 1; a.lo[1] = (int)(lo + n); a.hi[0] = (int)hi; a.hi[1] = n; }
    else if (hi > n) { a.count = 2; a.lo[0] = 1; a.lo[1] = (int)lo; a.hi[0] = (int)(hi - n); a.hi[1] = n; }
    else { a.count = 1; a.lo[0] = (int)lo; a.hi[0] = (int)hi; }
    return a;
}

static int valid_nucleus(const omodel* m, int x, int y, int z) {                          /* 3S:687-703, 2D:493-502 */
    const nicr_config* c = &m->c;
    const double r = c->radius_grid;
    if (x - r < 5. || x + r > (double)(c->nx - 3)) return 0;
    if (m->dim == 2) {
        const int sr = (int)ceil(r + c->exclusion_gap_grid);
        const int i0 = x - sr > 1 ? x - sr : 1, i1 = x + sr < c->nx ? x + sr : c->nx;
        for (int i = i0; i <= i1; ++i) for (int j = 1; j <= c->ny; ++j)
            if (A(m->p, i, j, 0) > .01 && hypot((double)(i - x), min_image(j - y, c->ny)) < r + c->exclusion_gap_grid) return 0;
        return 1;
    }
    const double limit = r + c->exclusion_gap_grid;
    const axis_nb ys = periodic_nb(y, limit, c->ny), zs = periodic_nb(z, limit, c->nz);
    const int sr = bounded_reach(limit, c->nx);
    const long long a0 = (long long)x - sr, a1 = (long long)x + sr;
    for (int i = (int)(a0 > 1 ? a0 : 1); i <= (int)(a1 < c->nx ? a1 : c->nx); ++i)
        for (int jy = 0; jy < ys.count; ++jy) for (int j = ys.lo[jy]; j <= ys.hi[jy]; ++j)
            for (int kz = 0; kz < zs.count; ++kz) for (int k = zs.lo[kz]; k <= zs.hi[kz]; ++k) {
                const double di = (double)(i - x), dj = min_image(j - y, c->ny), dk = min_image(k - z, c->nz);
                if (A(m->p, i, j, k) > .01 && sqrt(di * di + dj * dj + dk * dk) < r + c->exclusion_gap_grid) return 0;
            }
    return 1;
}

static void stamp_cell(omodel* m, int i, int j, int k) {
    m->b[B_NUCO] += PH_OXO - A(m->o, i, j, k); m->b[B_NUCCR] += PH_OXCR - A(m->cr, i, j, k);
    A(m->o, i, j, k) = PH_OXO; A(m->cr, i, j, k) = PH_OXCR; A(m->p, i, j, k) = 1.;
    for (int g = 0; g < m->neta; ++g) A(m->eta[g], i, j, k) = 0.;
}

int oracle_stamp(omodel* m, int x, int y, int z) {                                         /* 3S:704-724, 2D:503-516 */
    const nicr_config* c = &m->c;
    int changed = 0;
    if (m->dim == 2) {
        const int rr = (int)ceil(c->radius_grid);
        const int i0 = x - rr > 1 ? x - rr : 1, i1 = x + rr < c->nx ? x + rr : c->nx;
        for (int i = i0; i <= i1; ++i) for (int j = 1; j <= c->ny; ++j) {
            const double dy = min_image(j - y, c->ny);
            if ((i - x) * (i - x) + dy * dy <= c->radius_grid * c->radius_grid && A(m->p, i, j, 0) < .01) { stamp_cell(m, i, j, 0); ++changed; }
        }
        if (changed) ++m->nuclei;
        return changed;
    }
    const int rr = bounded_reach(c->radius_grid, c->nx);
    const axis_nb ys = periodic_nb(y, c->radius_grid, c->ny), zs = periodic_nb(z, c->radius_grid, c->nz);
    const long long a0 = (long long)x - rr, a1 = (long long)x + rr;
    for (int i = (int)(a0 > 1 ? a0 : 1); i <= (int)(a1 < c->nx ? a1 : c->nx); ++i)
        for (int jy = 0; jy < ys.count; ++jy) for (int j = ys.lo[jy]; j <= ys.hi[jy]; ++j)
            for (int kz = 0; kz < zs.count; ++kz) for (int k = zs.lo[kz]; k <= zs.hi[kz]; ++k) {
                const double dy = min_image(j - y, c->ny), dz = min_image(k - z, c->nz);
                if ((i - x) * (i - x) + dy * dy + dz * dz <= c->radius_grid * c->radius_grid && A(m->p, i, j, k) < .01) {
                    stamp_cell(m, i, j, k); ++changed;
                }
            }
    if (changed) { ++m->nuclei; if (m->has_eta) m->eta_dirty = 1; }
    return changed;
}

void oracle_nucleate(omodel* m) {                                                         /* 3S:752-759, 2D:543-550 */
    if (m->c.nucleation != NICR_NUC_KSP) return;
    FOR_CELLS(m) {
        if (A(m->p, i, j, k) <= .01 && A(m->o, i, j, k) * A(m->cr, i, j, k) > m->c.ksp && valid_nucleus(m, i, j, k))
            oracle_stamp(m, i, j, k);
    }
}

int oracle_run(omodel* m, int steps, int* done) {                                         /* 3S:1368-1385, 2D:1219-1236 */
    *done = 0;
    for (int s = 0; s < steps; ++s) {
        const long long n = m->steps_done + 1;
        const double time = n * m->c.dt;
        if (m->c.nucleation == NICR_NUC_KSP && time + 1.e-12 * m->c.nucleation_period >= m->next_nucleation) {
            oracle_nucleate(m);
            m->next_nucleation += m->c.nucleation_period;
        }
        const int rc = oracle_step(m);
        if (rc) return rc;
        ++*done;
    }
    return 0;
}

/* ---------------------------------------------------------------- diagnostics */
static void put_ld(double* out, long double v) { const double hi = (double)v; out[0] = hi; out[1] = (double)(v - (long double)hi); }

void oracle_budget(const omodel* m, double* hilo, long long* counts) {
    for (int q = 0; q < B_N; ++q) put_ld(hilo + 2 * q, m->b[q]);
    put_ld(hilo + 16, m->initialO); put_ld(hilo + 18, m->initialCr);
    counts[0] = m->nuclei; counts[1] = m->clipped;
}
void oracle_seeds(const omodel* m, double* xyz, long long* volumes) {
    const int D = m->dim;
    for (int g = 0; g < m->nseeds; ++g) {
        for (int d = 0; d < D; ++d) xyz[D * g + d] = m->seeds[D * g + d];
        volumes[g] = m->volumes[g];
    }
}
void oracle_log_values(omodel* m, double* out) {                                          /* 3S:963-977, 2D:697-710 */
    long double so = lsum(m, m->o), sc = lsum(m, m->cr), po = lsum(m, m->p), sumH = 0.;
    double omin = 1., omax = 0., crmin = 1., crmax = 0., nimin = 1., phimin = 1., phimax = 0.;
    FOR_CELLS(m) {
        const double o = A(m->o, i, j, k), cr = A(m->cr, i, j, k), p = A(m->p, i, j, k);
        sumH += h_(p);
        omin = smin(omin, o); omax = smax(omax, o); crmin = smin(crmin, cr); crmax = smax(crmax, cr);
        nimin = smin(nimin, 1. - o - cr); phimin = smin(phimin, p); phimax = smax(phimax, p);
    }
    put_ld(out, so); put_ld(out + 2, sc); put_ld(out + 4, po); put_ld(out + 6, sumH);
    out[8] = omin; out[9] = omax; out[10] = crmin; out[11] = crmax; out[12] = nimin; out[13] = phimin; out[14] = phimax;
}

static int current_grain(const omodel* m, int i, int j, int k) {                          /* 3S:527-533 */
    if (A(m->p, i, j, k) >= .5) return 0;
    if (!m->has_eta) return (int)A(m->grain, i, j, k);
    double best = 1.e-12; int id = 0;
    for (int g = 0; g < m->neta; ++g) if (A(m->eta[g], i, j, k) > best) { best = A(m->eta[g], i, j, k); id = g + 1; }
    return id;
}

static long double grain_energy(omodel* m) {                                              /* 3S:546-565, 2D:367-381 */
    const nicr_config* c = &m->c;
    long double local = 0.;
    if (!m->has_eta) return 0.;
    const double K = eta_K(c);
    FOR_CELLS(m) {
        double density;
        if (m->dim == 3) {
            double S = 0., pairs = 0.;
            for (int g = 0; g < m->neta; ++g) { const double q = A(m->eta[g], i, j, k) * A(m->eta[g], i, j, k); pairs += S * q; S += q; }
            density = g_energy(A(m->eta_s2, i, j, k), pairs, A(m->p, i, j, k), c);
        } else {
            density = g_energy(A(m->eta_s2, i, j, k), A(m->eta_pairs, i, j, k), A(m->p, i, j, k), c);
        }
        for (int g = 0; g < m->neta; ++g) {
            const double* e = m->eta[g];
            if (i < c->nx) { const double t = (A(e, i + 1, j, k) - A(e, i, j, k)) / c->dx; density += .5 * K * (t * t); }
            { const double t = (A(e, i, j + 1, k) - A(e, i, j, k)) / c->dy; density += .5 * K * (t * t); }
            if (m->dim == 3) { const double t = (A(e, i, j, k + 1) - A(e, i, j, k)) / c->dz; density += .5 * K * (t * t); }
        }
        local += m->dim == 3 ? density * c->dx * c->dy * c->dz : density * c->dx * c->dy;
    }
    return local;
}

int oracle_grain_values(omodel* m, double* out, long long* cells, double* amount) {     /* 3S:566-590, 2D:382-406 */
    if (!m->has_eta) return 1;
    oracle_refresh(m);
    const int N = m->neta;
    long double* amt = (long double*)calloc((size_t)N, sizeof(long double));
    for (int g = 0; g < N; ++g) cells[g] = 0;
    double lo = 1., hi = 0., slo = INFINITY, shi = 0., gbmax = 0.;
    long double sumS = 0., mask = 0.; long long unassigned = 0;
    FOR_CELLS(m) {
        const double S = A(m->eta_s2, i, j, k), metal = 1. - h_(A(m->p, i, j, k));
        slo = smin(slo, S); shi = smax(shi, S); sumS += S; mask += metal * A(m->gb, i, j, k); gbmax = smax(gbmax, A(m->gb, i, j, k));
        const int id = current_grain(m, i, j, k);
        if (id) ++cells[id - 1]; else if (A(m->p, i, j, k) < .5) ++unassigned;
        for (int g = 0; g < N; ++g) {
            const double v = A(m->eta[g], i, j, k);
            lo = smin(lo, v); hi = smax(hi, v);
            if (S > 1.e-24) amt[g] += metal * v * v / S;
        }
    }
    long long alive = 0;
    for (int g = 0; g < N; ++g) alive += cells[g] > 0;
    const long double energy = grain_energy(m);
    out[0] = lo; out[1] = hi; out[2] = slo; out[3] = shi;
    put_ld(out + 4, sumS); put_ld(out + 6, mask); put_ld(out + 8, energy);
    out[10] = gbmax; out[11] = (double)alive; out[12] = (double)unassigned;
    for (int g = 0; g < N; ++g) put_ld(amount + 2 * g, amt[g]);
    free(amt);
    return 0;
}
