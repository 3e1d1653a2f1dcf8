/*
 * synth.c -- seeded synthetic plenoptic raw frames (libpfd_synth.so).
 *
 * Stands in for the reference's raw_dataset/ captures, which are not available:
 *  - hexagonal micro-lens array, rows horizontal, odd rows offset by pitch/2,
 *    rows spaced pitch*sqrt(3)/2; tile key (column, row) as the white-image
 *    centre fit assigns them (DepthSolver.cpp:806-866);
 *  - lens types 0,1,2 interleaved so that the six ring neighbours of a lens
 *    have the other two types; each type has its own Gaussian blur sigma;
 *  - scene: n slanted planes in virtual depth v(X, Y) = c + a X + b Y, the
 *    nearest of n seeded sites chooses the plane (Voronoi), v clamped to
 *    [vd_min, vd_max]; texture: 4-octave value noise on (X, Y);
 *  - rendering: micro-image pixel u of lens c shows the virtual point
 *    X = c + (u - c) v(X) (LFRefocus::ComputeVirtual3D, FocalStack/LFRefocus.cpp:
 *    2100-2117), solved by fixed-point iteration; per-lens Gaussian blur,
 *    circular vignetting of radius pitch/2, additive Gaussian noise, rounding
 *    to 8 bits.
 * All randomness is a hash of (seed, purpose, index), so a frame is the same
 * on every machine with the same libm.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int width, height;
    float pitch;
    int n_planes;
    float vd_min, vd_max;
    float noise_sigma;
    int n_lens_types;
    float blur_sigma[3];
    float texture_cell;      /* base value-noise cell, virtual pixels (0 = 24) */
    uint64_t seed;
} pfd_synth_config;

static uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double u01(uint64_t seed, uint64_t a, uint64_t b)
{
    const uint64_t h = mix64(seed ^ mix64(a * 0x100000001B3ull + mix64(b)));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

typedef struct { double sx, sy, a, b, c; } plane_t;

static double lattice(uint64_t seed, int oct, long ix, long iy)
{
    return u01(seed, 0x7000 + (uint64_t)oct, ((uint64_t)(uint32_t)ix << 32) ^ (uint64_t)(uint32_t)iy);
}
static double smooth(double t) { return t * t * (3.0 - 2.0 * t); }
static double value_noise(uint64_t seed, double x, double y, double cell)
{
    double v = 0.0, amp = 1.0, norm = 0.0;
    for (int o = 0; o < 4; ++o) {
        const double fx = x / cell, fy = y / cell;
        const double x0 = floor(fx), y0 = floor(fy);
        const double tx = smooth(fx - x0), ty = smooth(fy - y0);
        const long ix = (long)x0, iy = (long)y0;
        const double a = lattice(seed, o, ix, iy), b = lattice(seed, o, ix + 1, iy);
        const double c = lattice(seed, o, ix, iy + 1), d = lattice(seed, o, ix + 1, iy + 1);
        v += amp * ((a + (b - a) * tx) * (1 - ty) + (c + (d - c) * tx) * ty);
        norm += amp;
        amp *= 0.5;
        cell *= 0.5;
    }
    return v / norm;
}

static double depth_at(const plane_t* P, int n, double vmin, double vmax, double X, double Y)
{
    int best = 0;
    double bd = 1e300;
    for (int i = 0; i < n; ++i) {
        const double dx = X - P[i].sx, dy = Y - P[i].sy, d = dx * dx + dy * dy;
        if (d < bd) { bd = d; best = i; }
    }
    double v = P[best].c + P[best].a * (X - P[best].sx) + P[best].b * (Y - P[best].sy);
    if (v < vmin) v = vmin;
    if (v > vmax) v = vmax;
    return v;
}

static void lens_grid(const pfd_synth_config* c, int* ncols, int* nrows, double* x0, double* y0, double* dy)
{
    const double p = c->pitch;
    *dy = p * sqrt(3.0) / 2.0;
    *x0 = 0.5 * p + 0.37;
    *y0 = 0.5 * p + 0.21;
    *nrows = (int)floor((c->height - 0.5 * p - *y0) / *dy) + 1;
    *ncols = (int)floor((c->width - 0.5 * p - *x0 - 0.5 * p) / p) + 1;   /* fits odd rows too */
    if (*nrows < 0) *nrows = 0;
    if (*ncols < 0) *ncols = 0;
}

int pfd_synth_count(const pfd_synth_config* c, int* n_lenses, int* n_cols, int* n_rows)
{
    if (!c || c->width <= 0 || c->height <= 0 || !(c->pitch > 2.0f)) return -1;
    int nc, nr;
    double x0, y0, dy;
    lens_grid(c, &nc, &nr, &x0, &y0, &dy);
    if (n_lenses) *n_lenses = nc * nr;
    if (n_cols) *n_cols = nc;
    if (n_rows) *n_rows = nr;
    return 0;
}

/* raw: width*height bytes; centers [L][2]; keys [L][2] (col,row); types [L];
 * vd_center [L] (ground-truth virtual depth at the lens centre).  Lenses in
 * key order (row-major). */
int pfd_synth_render(const pfd_synth_config* c, uint8_t* raw, float* centers, int* keys, int* types, float* vd_center)
{
    int nc, nr;
    double x0, y0, dy;
    if (!c || !raw || c->n_planes < 1 || c->n_planes > 4096 || !(c->pitch > 2.0f)) return -1;
    lens_grid(c, &nc, &nr, &x0, &y0, &dy);
    const int W = c->width, H = c->height, L = nc * nr;
    const double p = c->pitch, R = 0.5 * p;
    const double vmin = c->vd_min, vmax = c->vd_max;
    const double cell = c->texture_cell > 0 ? c->texture_cell : 24.0;
    const int ntypes = c->n_lens_types < 1 ? 1 : (c->n_lens_types > 3 ? 3 : c->n_lens_types);

    plane_t* P = (plane_t*)malloc(sizeof(plane_t) * (size_t)c->n_planes);
    if (!P) return -2;
    const double g = 3.0 / (double)(W > H ? W : H);
    for (int i = 0; i < c->n_planes; ++i) {
        P[i].sx = u01(c->seed, 1, i) * W;
        P[i].sy = u01(c->seed, 2, i) * H;
        P[i].a = (2.0 * u01(c->seed, 3, i) - 1.0) * g;
        P[i].b = (2.0 * u01(c->seed, 4, i) - 1.0) * g;
        P[i].c = vmin + 1.0 + u01(c->seed, 5, i) * (vmax - vmin - 2.0);
    }
    memset(raw, 0, (size_t)W * H);

#pragma omp parallel for schedule(dynamic, 8)
    for (int l = 0; l < L; ++l) {
        const int row = l / nc, col = l % nc;
        const double cx = x0 + col * p + ((row & 1) ? 0.5 * p : 0.0);
        const double cy = y0 + row * dy;
        const int type = (col + 2 * (row & 1) + ((row >> 1) & 1) * 0) % ntypes;
        if (centers) { centers[2 * l] = (float)cx; centers[2 * l + 1] = (float)cy; }
        if (keys) { keys[2 * l] = col; keys[2 * l + 1] = row; }
        if (types) types[l] = type;
        if (vd_center) vd_center[l] = (float)depth_at(P, c->n_planes, vmin, vmax, cx, cy);

        const double sigma = c->blur_sigma[type];
        const int br = sigma > 0 ? (int)ceil(3.0 * sigma) : 0;
        const int half = (int)ceil(R) + br + 1;
        const int side = 2 * half + 1;
        double* buf = (double*)malloc(sizeof(double) * side * side * 2);
        if (!buf) continue;
        double* tmp = buf + side * side;
        const int ox = (int)floor(cx) - half, oy = (int)floor(cy) - half;
        for (int j = 0; j < side; ++j)
            for (int i = 0; i < side; ++i) {
                const double ux = ox + i, uy = oy + j;
                double X = cx, Y = cy;
                for (int it = 0; it < 8; ++it) {
                    const double v = depth_at(P, c->n_planes, vmin, vmax, X, Y);
                    X = cx + (ux - cx) * v;
                    Y = cy + (uy - cy) * v;
                }
                buf[j * side + i] = 30.0 + 200.0 * value_noise(c->seed, X, Y, cell);
            }
        if (br > 0) {
            double k[64];
            double ks = 0.0;
            for (int t = -br; t <= br; ++t) { k[t + br] = exp(-0.5 * t * t / (sigma * sigma)); ks += k[t + br]; }
            for (int t = 0; t <= 2 * br; ++t) k[t] /= ks;
            for (int j = 0; j < side; ++j)
                for (int i = 0; i < side; ++i) {
                    double s = 0.0;
                    for (int t = -br; t <= br; ++t) {
                        int ii = i + t; ii = ii < 0 ? 0 : (ii >= side ? side - 1 : ii);
                        s += k[t + br] * buf[j * side + ii];
                    }
                    tmp[j * side + i] = s;
                }
            for (int j = 0; j < side; ++j)
                for (int i = 0; i < side; ++i) {
                    double s = 0.0;
                    for (int t = -br; t <= br; ++t) {
                        int jj = j + t; jj = jj < 0 ? 0 : (jj >= side ? side - 1 : jj);
                        s += k[t + br] * tmp[jj * side + i];
                    }
                    buf[j * side + i] = s;
                }
        }
        for (int j = 0; j < side; ++j)
            for (int i = 0; i < side; ++i) {
                const int ux = ox + i, uy = oy + j;
                if (ux < 0 || uy < 0 || ux >= W || uy >= H) continue;
                const double r = sqrt((ux - cx) * (ux - cx) + (uy - cy) * (uy - cy));
                if (r >= R) continue;
                double vig = 1.0;
                if (r > 0.9 * R) vig = 0.5 + 0.5 * cos(3.14159265358979323846 * (r - 0.9 * R) / (0.1 * R));
                double val = buf[j * side + i] * (0.75 + 0.25 * vig);
                if (c->noise_sigma > 0) {
                    const uint64_t pix = (uint64_t)uy * (uint64_t)W + (uint64_t)ux;
                    const double a = u01(c->seed, 11, pix), b = u01(c->seed, 12, pix);
                    const double n = sqrt(-2.0 * log(a + 1e-300)) * cos(2.0 * 3.14159265358979323846 * b);
                    val += c->noise_sigma * n;
                }
                long q = lround(val);
                raw[(size_t)uy * W + ux] = (uint8_t)(q < 0 ? 0 : (q > 255 ? 255 : q));
            }
        free(buf);
    }
    free(P);
    return 0;
}

/* Ground truth of a frame: vd_map (width*height floats) receives, at every raw
 * pixel inside a lens's circle, the virtual depth v of the scene point that
 * pixel shows (the same fixed point X = c + (u - c) v(X) the rendering solves),
 * and 0 elsewhere.  Lens circles of radius pitch/2 on the hexagonal grid touch
 * but do not overlap, so each pixel has one lens.  Since a neighbour lens at
 * baseline b sees that point shifted by b / v, the matched disparity of the
 * pixel against a neighbour one pitch away is pitch / v. */
int pfd_synth_vd_map(const pfd_synth_config* c, float* vd_map)
{
    int nc, nr;
    double x0, y0, dy;
    if (!c || !vd_map || c->n_planes < 1 || c->n_planes > 4096 || !(c->pitch > 2.0f)) return -1;
    lens_grid(c, &nc, &nr, &x0, &y0, &dy);
    const int W = c->width, H = c->height, L = nc * nr;
    const double p = c->pitch, R = 0.5 * p;
    const double vmin = c->vd_min, vmax = c->vd_max;
    plane_t* P = (plane_t*)malloc(sizeof(plane_t) * (size_t)c->n_planes);
    if (!P) return -2;
    const double g = 3.0 / (double)(W > H ? W : H);
    for (int i = 0; i < c->n_planes; ++i) {
        P[i].sx = u01(c->seed, 1, i) * W;
        P[i].sy = u01(c->seed, 2, i) * H;
        P[i].a = (2.0 * u01(c->seed, 3, i) - 1.0) * g;
        P[i].b = (2.0 * u01(c->seed, 4, i) - 1.0) * g;
        P[i].c = vmin + 1.0 + u01(c->seed, 5, i) * (vmax - vmin - 2.0);
    }
    memset(vd_map, 0, sizeof(float) * (size_t)W * H);
#pragma omp parallel for schedule(dynamic, 8)
    for (int l = 0; l < L; ++l) {
        const int row = l / nc, col = l % nc;
        const double cx = x0 + col * p + ((row & 1) ? 0.5 * p : 0.0);
        const double cy = y0 + row * dy;
        const int half = (int)ceil(R) + 1;
        const int ox = (int)floor(cx) - half, oy = (int)floor(cy) - half;
        for (int j = 0; j <= 2 * half; ++j)
            for (int i = 0; i <= 2 * half; ++i) {
                const int ux = ox + i, uy = oy + j;
                if (ux < 0 || uy < 0 || ux >= W || uy >= H) continue;
                const double r = sqrt((ux - cx) * (ux - cx) + (uy - cy) * (uy - cy));
                if (r >= R) continue;
                double X = cx, Y = cy, v = 0.0;
                for (int it = 0; it < 8; ++it) {
                    v = depth_at(P, c->n_planes, vmin, vmax, X, Y);
                    X = cx + (ux - cx) * v;
                    Y = cy + (uy - cy) * v;
                }
                vd_map[(size_t)uy * W + ux] = (float)depth_at(P, c->n_planes, vmin, vmax, X, Y);
            }
    }
    free(P);
    return 0;
}
