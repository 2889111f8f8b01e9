/*
 * fn_generate.cpp -- seeded placement of straight fibres for the synthetic
 * workloads (the reference ships no model files).  Host-only code.
 *
 * Each fibre is `beads` beads `spacing` apart along a random direction
 * (uniform in the xy plane with a uniform z tilt, or uniform on the sphere);
 * its centre is uniform in the box with z in [zlo, zhi].  On finite axes the
 * fibre is redrawn until it lies inside the box.  With min_sep > 0 every bead
 * keeps that distance from the beads already placed (minimum image on
 * periodic axes): for a drawn (x, y, direction) the centre height is drawn
 * uniformly from the heights that satisfy it, and the draw is repeated when
 * none does.  The random stream is xoshiro256** seeded through splitmix64.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/fibrenet_generate.h"

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (int i = 0; i < 4; ++i) {
            seed += 0x9e3779b97f4a7c15ull;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
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
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
};

void direction(Rng& rng, double tilt_deg, int orient, double d[3]) {
    const double two_pi = 6.283185307179586;
    if (orient == 1) {
        const double z = rng.uniform(-1.0, 1.0);
        const double phi = rng.uniform(0.0, two_pi);
        const double r = std::sqrt(std::max(0.0, 1.0 - z * z));
        d[0] = r * std::cos(phi);
        d[1] = r * std::sin(phi);
        d[2] = z;
        return;
    }
    const double phi = rng.uniform(0.0, two_pi);
    const double tilt = rng.uniform(-tilt_deg, tilt_deg) * (3.141592653589793 / 180.0);
    d[0] = std::cos(phi) * std::cos(tilt);
    d[1] = std::sin(phi) * std::cos(tilt);
    d[2] = std::sin(tilt);
}

}  // namespace

static int place_fibres(unsigned long long seed, int n_fibres, int beads, const double box[3],
                        int periodic_mask, double zlo, double zhi, double tilt_deg, int orient,
                        double spacing, double min_sep, int max_tries, double* out);

/* fn_place_fibres behind a guard: host memory running out returns 3 instead
   of an exception crossing the C ABI. */
extern "C" FN_GEN_API int fn_place_fibres(unsigned long long seed, int n_fibres, int beads,
                                          const double box[3], int periodic_mask, double zlo,
                                          double zhi, double tilt_deg, int orient, double spacing,
                                          double min_sep, int max_tries, double* out) {
    try {
        return place_fibres(seed, n_fibres, beads, box, periodic_mask, zlo, zhi, tilt_deg, orient,
                            spacing, min_sep, max_tries, out);
    } catch (const std::exception&) {
        return 3;
    }
}

static int place_fibres(unsigned long long seed, int n_fibres, int beads, const double box[3],
                        int periodic_mask, double zlo, double zhi, double tilt_deg, int orient,
                        double spacing, double min_sep, int max_tries, double* out) {
    if (n_fibres < 0 || beads <= 0 || !box || !out || max_tries <= 0) return 1;
    Rng rng(seed);
    const bool per[3] = {(periodic_mask & 1) != 0, (periodic_mask & 2) != 0, (periodic_mask & 4) != 0};
    std::vector<double> off(beads);
    for (int b = 0; b < beads; ++b) off[b] = (b - (beads - 1) / 2.0) * spacing;
    const double r2 = min_sep * min_sep;
    int ncx = 1, ncy = 1;
    double cw[2] = {box[0], box[1]};
    std::vector<std::vector<double>> cols;
    if (min_sep > 0.0) {
        ncx = std::max(1, (int)(box[0] / min_sep));
        ncy = std::max(1, (int)(box[1] / min_sep));
        cw[0] = box[0] / ncx;
        cw[1] = box[1] / ncy;
        cols.resize((size_t)ncx * ncy);
    }
    std::vector<double> pts(3 * (size_t)beads), rel(3 * (size_t)beads);
    std::vector<std::pair<double, double>> iv;
    for (int f = 0; f < n_fibres; ++f) {
        bool placed = false;
        for (int tr = 0; tr < max_tries && !placed; ++tr) {
            double c[3] = {rng.uniform() * box[0], rng.uniform() * box[1], rng.uniform(zlo, zhi)};
            double d[3];
            direction(rng, tilt_deg, orient, d);
            double zmin = 1e300, zmax = -1e300;
            bool bad = false;
            for (int b = 0; b < beads; ++b) {
                for (int a = 0; a < 3; ++a) {
                    rel[3 * b + a] = off[b] * d[a];
                    pts[3 * b + a] = c[a] + rel[3 * b + a];
                }
                zmin = std::min(zmin, rel[3 * b + 2]);
                zmax = std::max(zmax, rel[3 * b + 2]);
                for (int a = 0; a < 2; ++a)
                    if (!per[a] && (pts[3 * b + a] < 0.0 || pts[3 * b + a] > box[a])) bad = true;
            }
            if (bad) continue;
            if (min_sep <= 0.0) {
                if (!per[2]) {
                    for (int b = 0; b < beads && !bad; ++b)
                        if (pts[3 * b + 2] < 0.0 || pts[3 * b + 2] > box[2]) bad = true;
                    if (bad) continue;
                }
                placed = true;
                break;
            }
            double lo = std::max(zlo - zmin, zlo), hi = std::min(zhi - zmax, zhi);
            if (!per[2]) {
                lo = std::max(lo, -zmin);
                hi = std::min(hi, box[2] - zmax);
            }
            if (!(hi > lo)) continue;
            iv.clear();
            for (int b = 0; b < beads; ++b) {
                const int ix = (int)std::floor(pts[3 * b] / cw[0]);
                const int iy = (int)std::floor(pts[3 * b + 1] / cw[1]);
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy) {
                        int jx = ix + dx, jy = iy + dy;
                        if (per[0]) jx = ((jx % ncx) + ncx) % ncx;
                        else if (jx < 0 || jx >= ncx) continue;
                        if (per[1]) jy = ((jy % ncy) + ncy) % ncy;
                        else if (jy < 0 || jy >= ncy) continue;
                        const std::vector<double>& col = cols[(size_t)jx * ncy + jy];
                        for (size_t q = 0; q < col.size(); q += 3) {
                            double ddx = col[q] - pts[3 * b], ddy = col[q + 1] - pts[3 * b + 1];
                            if (per[0]) ddx -= box[0] * std::nearbyint(ddx / box[0]);
                            if (per[1]) ddy -= box[1] * std::nearbyint(ddy / box[1]);
                            const double qq = ddx * ddx + ddy * ddy;
                            if (qq < r2) {
                                const double h = std::sqrt(r2 - qq);
                                const double zc = col[q + 2] - rel[3 * b + 2];
                                iv.emplace_back(zc - h, zc + h);
                                if (per[2]) {
                                    iv.emplace_back(zc - h - box[2], zc + h - box[2]);
                                    iv.emplace_back(zc - h + box[2], zc + h + box[2]);
                                }
                            }
                        }
                    }
            }
            std::sort(iv.begin(), iv.end());
            std::vector<std::pair<double, double>> freeseg;
            double cur = lo;
            for (auto& p : iv) {
                if (p.first > cur) freeseg.emplace_back(cur, std::min(p.first, hi));
                cur = std::max(cur, p.second);
                if (cur >= hi) break;
            }
            if (cur < hi) freeseg.emplace_back(cur, hi);
            double total = 0.0;
            for (auto& s : freeseg)
                if (s.second > s.first) total += s.second - s.first;
            if (!(total > 0.0)) continue;
            double u = rng.uniform() * total;
            double zc = lo;
            for (auto& s : freeseg) {
                const double len = s.second - s.first;
                if (!(len > 0.0)) continue;
                if (u <= len) {
                    zc = s.first + u;
                    break;
                }
                u -= len;
                zc = s.second;
            }
            for (int b = 0; b < beads; ++b) pts[3 * b + 2] = zc + rel[3 * b + 2];
            placed = true;
        }
        if (!placed) return 2;
        for (int b = 0; b < beads; ++b) {
            for (int a = 0; a < 3; ++a) out[((size_t)f * beads + b) * 3 + a] = pts[3 * b + a];
            if (min_sep > 0.0) {
                double w[3];
                for (int a = 0; a < 3; ++a) {
                    w[a] = pts[3 * b + a];
                    if (per[a]) w[a] -= box[a] * std::floor(w[a] / box[a]);
                }
                const int jx = std::min(ncx - 1, std::max(0, (int)std::floor(w[0] / cw[0])));
                const int jy = std::min(ncy - 1, std::max(0, (int)std::floor(w[1] / cw[1])));
                std::vector<double>& col = cols[(size_t)jx * ncy + jy];
                col.push_back(w[0]);
                col.push_back(w[1]);
                col.push_back(w[2]);
            }
        }
    }
    return 0;
}
