// synth.cpp -- seeded synthetic binary images and volumes of the workload
// shapes: Bezier strokes (512x512 frames, batched images, serving frames),
// vessel-like 2D trees with salt and holes (4096x4096), tubular 3D trees with
// solid ellipsoids (volumes).  Host C++, no CUDA; built as libbgt_synth.so.
//
// Every generator is a pure function of its seed (splitmix64 seeding a
// xoshiro256** stream), clears the outer 1-pixel/voxel frame (the
// reference's precondition: no foreground on the image border), and writes
// uint8 {0,1}.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t &x)
    {
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed)
    {
        uint64_t x = seed;
        for (auto &v : s) v = splitmix(x);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next()
    {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uni(double a, double b) { return a + (b - a) * uni(); }
};

constexpr double kPi = 3.14159265358979323846;

struct Img2 {
    int w, h;
    uint8_t *p;
    void disc(double cx, double cy, double r, uint8_t v = 1)
    {
        const int x0 = std::max(0, (int)std::floor(cx - r)), x1 = std::min(w - 1, (int)std::ceil(cx + r));
        const int y0 = std::max(0, (int)std::floor(cy - r)), y1 = std::min(h - 1, (int)std::ceil(cy + r));
        const double r2 = r * r;
        for (int y = y0; y <= y1; y++) {
            const double dy = y - cy;
            for (int x = x0; x <= x1; x++) {
                const double dx = x - cx;
                if (dx * dx + dy * dy <= r2) p[(size_t)y * w + x] = v;
            }
        }
    }
    void clear_frame()
    {
        for (int x = 0; x < w; x++) p[x] = p[(size_t)(h - 1) * w + x] = 0;
        for (int y = 0; y < h; y++) p[(size_t)y * w] = p[(size_t)y * w + w - 1] = 0;
    }
};

struct Img3 {
    int w, h, d;
    uint8_t *p;
    void sphere(double cx, double cy, double cz, double r)
    {
        const int x0 = std::max(0, (int)std::floor(cx - r)), x1 = std::min(w - 1, (int)std::ceil(cx + r));
        const int y0 = std::max(0, (int)std::floor(cy - r)), y1 = std::min(h - 1, (int)std::ceil(cy + r));
        const int z0 = std::max(0, (int)std::floor(cz - r)), z1 = std::min(d - 1, (int)std::ceil(cz + r));
        const double r2 = r * r;
        for (int z = z0; z <= z1; z++)
            for (int y = y0; y <= y1; y++) {
                const double dz = z - cz, dy = y - cy;
                for (int x = x0; x <= x1; x++) {
                    const double dx = x - cx;
                    if (dx * dx + dy * dy + dz * dz <= r2) p[((size_t)z * h + y) * w + x] = 1;
                }
            }
    }
    void clear_frame()
    {
        for (int z = 0; z < d; z++)
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++)
                    if (z == 0 || y == 0 || x == 0 || z == d - 1 || y == h - 1 || x == w - 1)
                        p[((size_t)z * h + y) * w + x] = 0;
    }
};

// Cubic Bezier from 4 control points, discs at >= 2 samples per pixel of arc length.
void draw_bezier(Img2 &im, const double *c, double r)
{
    auto at = [&](double t, double &x, double &y) {
        const double u = 1 - t;
        const double b0 = u * u * u, b1 = 3 * u * u * t, b2 = 3 * u * t * t, b3 = t * t * t;
        x = b0 * c[0] + b1 * c[2] + b2 * c[4] + b3 * c[6];
        y = b0 * c[1] + b1 * c[3] + b2 * c[5] + b3 * c[7];
    };
    double len = 0, px, py;
    at(0, px, py);
    for (int i = 1; i <= 64; i++) {
        double x, y;
        at(i / 64.0, x, y);
        len += std::hypot(x - px, y - py);
        px = x;
        py = y;
    }
    const int n = std::max(2, (int)std::ceil(2 * len) + 1);
    for (int i = 0; i < n; i++) {
        double x, y;
        at((double)i / (n - 1), x, y);
        im.disc(x, y, r);
    }
}

void draw_segment2(Img2 &im, double x0, double y0, double x1, double y1, double r0, double r1)
{
    const double len = std::hypot(x1 - x0, y1 - y0);
    const int n = std::max(2, (int)std::ceil(2 * len) + 1);
    for (int i = 0; i < n; i++) {
        const double t = (double)i / (n - 1);
        im.disc(x0 + t * (x1 - x0), y0 + t * (y1 - y0), r0 + t * (r1 - r0));
    }
}

void draw_segment3(Img3 &im, const double *a, const double *b, double r0, double r1)
{
    const double len = std::sqrt((b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) +
                                 (b[2] - a[2]) * (b[2] - a[2]));
    const int n = std::max(2, (int)std::ceil(2 * len) + 1);
    for (int i = 0; i < n; i++) {
        const double t = (double)i / (n - 1);
        im.sphere(a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1]), a[2] + t * (b[2] - a[2]),
                  r0 + t * (r1 - r0));
    }
}

// 2D binary tree: branch of length U[lmin,lmax] from (x,y) at angle ang;
// children at ang +/- U[amin,amax]; radius tapers linearly with depth.
void tree2(Img2 &im, Rng &g, double x, double y, double ang, int level, int depth, double lmin,
           double lmax, double amin, double amax, double r0, double r1)
{
    const double len = g.uni(lmin, lmax);
    const double x1 = x + len * std::cos(ang), y1 = y + len * std::sin(ang);
    const double ra = r0 + (r1 - r0) * level / depth, rb = r0 + (r1 - r0) * (level + 1) / depth;
    draw_segment2(im, x, y, x1, y1, ra, rb);
    if (level + 1 >= depth) return;
    const double da = g.uni(amin, amax), db = g.uni(amin, amax);
    tree2(im, g, x1, y1, ang + da, level + 1, depth, lmin, lmax, amin, amax, r0, r1);
    tree2(im, g, x1, y1, ang - db, level + 1, depth, lmin, lmax, amin, amax, r0, r1);
}

void unit3(Rng &g, double *v)
{
    for (;;) {
        v[0] = g.uni(-1, 1);
        v[1] = g.uni(-1, 1);
        v[2] = g.uni(-1, 1);
        const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (n > 1e-3 && n <= 1) {
            v[0] /= n; v[1] /= n; v[2] /= n;
            return;
        }
    }
}

// rotate unit vector v by angle a towards a random perpendicular direction
void tilt(Rng &g, const double *v, double a, double *out)
{
    double r[3], p[3];
    unit3(g, r);
    const double dot = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
    for (int k = 0; k < 3; k++) p[k] = r[k] - dot * v[k];
    const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    if (n < 1e-6) {
        for (int k = 0; k < 3; k++) out[k] = v[k];
        return;
    }
    for (int k = 0; k < 3; k++) out[k] = std::cos(a) * v[k] + std::sin(a) * p[k] / n;
}

void tree3(Img3 &im, Rng &g, const double *x, const double *dir, int level, int depth, double lmin,
           double lmax, double amin, double amax, double r0, double r1)
{
    const double len = g.uni(lmin, lmax);
    double e[3] = {x[0] + len * dir[0], x[1] + len * dir[1], x[2] + len * dir[2]};
    const double ra = r0 + (r1 - r0) * level / depth, rb = r0 + (r1 - r0) * (level + 1) / depth;
    draw_segment3(im, x, e, ra, rb);
    if (level + 1 >= depth) return;
    double d1[3], d2[3];
    tilt(g, dir, g.uni(amin, amax), d1);
    tilt(g, dir, g.uni(amin, amax), d2);
    tree3(im, g, e, d1, level + 1, depth, lmin, lmax, amin, amax, r0, r1);
    tree3(im, g, e, d2, level + 1, depth, lmin, lmax, amin, amax, r0, r1);
}

}  // namespace

extern "C" {

// Uniform doubles in [0,1) from the generator stream of `seed` (lets callers
// derive batch shapes and stream parameters from the same seed family).
void bgt_synth_uniform(uint64_t seed, int64_t n, double *out)
{
    Rng g(seed);
    for (int64_t i = 0; i < n; i++) out[i] = g.uni();
}

// Explicit strokes: ctrl = n x 8 doubles (x0,y0,...,x3,y3), radius = n.
// Writes into out (w*h), which the caller zeroes; clears the frame.
void bgt_synth_render_strokes2d(int w, int h, int n, const double *ctrl, const double *radius, uint8_t *out)
{
    Img2 im{w, h, out};
    for (int i = 0; i < n; i++) draw_bezier(im, ctrl + 8 * i, radius[i]);
    im.clear_frame();
}

// n random cubic Bezier strokes, control points uniform in the frame, radius U[rmin,rmax].
void bgt_synth_strokes2d(uint64_t seed, int w, int h, int n, double rmin, double rmax, uint8_t *out)
{
    std::memset(out, 0, (size_t)w * h);
    Rng g(seed);
    Img2 im{w, h, out};
    double c[8];
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < 4; k++) {
            c[2 * k] = g.uni(0, w);
            c[2 * k + 1] = g.uni(0, h);
        }
        draw_bezier(im, c, g.uni(rmin, rmax));
    }
    im.clear_frame();
}

// Vessel-like trees: nroots roots uniform in the frame, binary branching to
// `depth` levels, branch length U[lmin,lmax], child angle +/-U[amin,amax]
// degrees, radius r0 -> r1 over the depth; then salt (a fraction of pixels set
// to 1 at uniform positions) and nholes elliptical holes (semi-axes
// U[hmin,hmax], random angle) set to 0.
void bgt_synth_vessels2d(uint64_t seed, int w, int h, int nroots, int depth, double lmin, double lmax,
                         double amin_deg, double amax_deg, double r0, double r1, double salt,
                         int nholes, double hmin, double hmax, uint8_t *out)
{
    std::memset(out, 0, (size_t)w * h);
    Rng g(seed);
    Img2 im{w, h, out};
    const double amin = amin_deg * kPi / 180, amax = amax_deg * kPi / 180;
    for (int i = 0; i < nroots; i++) {
        const double x = g.uni(0, w), y = g.uni(0, h), a = g.uni(0, 2 * kPi);
        tree2(im, g, x, y, a, 0, depth, lmin, lmax, amin, amax, r0, r1);
    }
    const int64_t nsalt = (int64_t)std::llround(salt * (double)w * h);
    for (int64_t i = 0; i < nsalt; i++) {
        const int x = (int)(g.uni() * w), y = (int)(g.uni() * h);
        out[(size_t)y * w + x] = 1;
    }
    for (int i = 0; i < nholes; i++) {
        const double cx = g.uni(0, w), cy = g.uni(0, h);
        const double a = g.uni(hmin, hmax), b = g.uni(hmin, hmax), th = g.uni(0, kPi);
        const double ct = std::cos(th), st = std::sin(th), R = std::max(a, b);
        for (int y = std::max(0, (int)(cy - R) - 1); y <= std::min(h - 1, (int)(cy + R) + 1); y++)
            for (int x = std::max(0, (int)(cx - R) - 1); x <= std::min(w - 1, (int)(cx + R) + 1); x++) {
                const double dx = x - cx, dy = y - cy;
                const double u = (ct * dx + st * dy) / a, v = (-st * dx + ct * dy) / b;
                if (u * u + v * v <= 1) out[(size_t)y * w + x] = 0;
            }
    }
    im.clear_frame();
}

// Tubular 3D trees (roots uniform, initial direction uniform on the sphere,
// binary branching to `depth` levels, length U[lmin,lmax], child tilt
// U[amin,amax] degrees, radius r0 -> r1, spheres swept along each branch)
// plus nell solid ellipsoids (semi-axes U[emin,emax], random rotation).
void bgt_synth_trees3d(uint64_t seed, int w, int h, int d, int ntrees, int depth, double lmin, double lmax,
                       double amin_deg, double amax_deg, double r0, double r1, int nell, double emin,
                       double emax, uint8_t *out)
{
    std::memset(out, 0, (size_t)w * h * d);
    Rng g(seed);
    Img3 im{w, h, d, out};
    const double amin = amin_deg * kPi / 180, amax = amax_deg * kPi / 180;
    for (int i = 0; i < ntrees; i++) {
        double x[3] = {g.uni(0, w), g.uni(0, h), g.uni(0, d)}, dir[3];
        unit3(g, dir);
        tree3(im, g, x, dir, 0, depth, lmin, lmax, amin, amax, r0, r1);
    }
    for (int i = 0; i < nell; i++) {
        const double c[3] = {g.uni(0, w), g.uni(0, h), g.uni(0, d)};
        const double ax[3] = {g.uni(emin, emax), g.uni(emin, emax), g.uni(emin, emax)};
        // random orthonormal frame (Gram-Schmidt on two random unit vectors)
        double e0[3], e1[3], e2[3];
        unit3(g, e0);
        unit3(g, e1);
        const double dd = e0[0] * e1[0] + e0[1] * e1[1] + e0[2] * e1[2];
        for (int k = 0; k < 3; k++) e1[k] -= dd * e0[k];
        const double n1 = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
        for (int k = 0; k < 3; k++) e1[k] /= n1;
        e2[0] = e0[1] * e1[2] - e0[2] * e1[1];
        e2[1] = e0[2] * e1[0] - e0[0] * e1[2];
        e2[2] = e0[0] * e1[1] - e0[1] * e1[0];
        const double R = std::max(ax[0], std::max(ax[1], ax[2]));
        for (int z = std::max(0, (int)(c[2] - R) - 1); z <= std::min(d - 1, (int)(c[2] + R) + 1); z++)
            for (int y = std::max(0, (int)(c[1] - R) - 1); y <= std::min(h - 1, (int)(c[1] + R) + 1); y++)
                for (int x = std::max(0, (int)(c[0] - R) - 1); x <= std::min(w - 1, (int)(c[0] + R) + 1); x++) {
                    const double p[3] = {x - c[0], y - c[1], z - c[2]};
                    const double u = (p[0] * e0[0] + p[1] * e0[1] + p[2] * e0[2]) / ax[0];
                    const double v = (p[0] * e1[0] + p[1] * e1[1] + p[2] * e1[2]) / ax[1];
                    const double q = (p[0] * e2[0] + p[1] * e2[1] + p[2] * e2[2]) / ax[2];
                    if (u * u + v * v + q * q <= 1) out[((size_t)z * h + y) * w + x] = 1;
                }
    }
    im.clear_frame();
}

}  // extern "C"
