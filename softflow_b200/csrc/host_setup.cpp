// host_setup.cpp -- host-side setup helpers of the C ABI: circular capsule
// rest geometry and seeded rejection placement.  Setup-time FP64 host code
// (the reference runs these in the Capsule constructor and
// Simulation::addCapsuleRandom); nothing here runs per step.
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "../../include/softflow_gpu.h"

namespace sfg_host {
void set_error(const std::string& msg);
}

namespace {

constexpr double kPi = 3.14159265358979323846;

struct V2 {
    double x, y;
};
inline V2 sub(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
inline double nrm(V2 a) { return std::sqrt(a.x * a.x + a.y * a.y); }
inline double crs(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }
inline double dt(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }

// Capsule::computeOptimalNodes (capsule.h:14-17)
int optimal_nodes(double radius) {
    int n = static_cast<int>(std::ceil(2.0 * kPi * radius / 0.75));
    return n > 12 ? n : 12;
}

// Rest geometry of a circle (capsule.cpp:7-141 for CapsuleShape::CIRCLE).
// Built with periodic_nx = 0 as in the reference, where the periodic flag is
// applied only after construction (capsule_system.cpp:5-9).
void build_circle(double cx, double cy, double radius, int nn, const sfg_membrane_params& mp,
                  sfg_capsule_rest& rest, std::vector<V2>& P, std::vector<double>& L0,
                  std::vector<double>& ang, std::vector<double>& ds) {
    P.resize(nn);
    L0.resize(nn);
    ang.assign(nn, 0.0);
    ds.assign(nn, 0.0);
    for (int i = 0; i < nn; ++i) {
        const double th = 2.0 * kPi * i / nn;
        P[i] = {cx + radius * std::cos(th), cy + radius * std::sin(th)};
    }
    for (int i = 0; i < nn; ++i) L0[i] = nrm(sub(P[(i + 1) % nn], P[i]));
    double A = 0.0, Pm = 0.0;
    for (int i = 0; i < nn; ++i) A += crs(P[i], P[(i + 1) % nn]);
    for (int i = 0; i < nn; ++i) Pm += nrm(sub(P[(i + 1) % nn], P[i]));
    rest.num_nodes = nn;
    rest.rest_area = 0.5 * std::abs(A);
    rest.rest_perimeter = Pm;
    rest.wlc_kBT_p = mp.wlc_kBT_p;
    rest.wlc_k_pow = mp.wlc_k_pow;
    if (mp.model == SFG_WLC && nn > 0) {
        const double l0 = L0[0];
        const double L_max = mp.wlc_L_max_ratio * l0;
        const double x0 = l0 / L_max;
        if (rest.wlc_kBT_p <= 0.0) {
            const double denom = 1.0 / (2.0 * (1.0 - x0) * (1.0 - x0) * (1.0 - x0)) + 1.0;
            rest.wlc_kBT_p = mp.G_s * L_max / (l0 * denom);
        }
        if (rest.wlc_k_pow <= 0.0) {
            const double F_rest = rest.wlc_kBT_p * (1.0 / (4.0 * (1.0 - x0) * (1.0 - x0)) - 0.25 + x0);
            rest.wlc_k_pow = F_rest * l0;
        }
    }
    if (mp.use_helfrich) {
        for (int i = 0; i < nn; ++i) {
            const V2 ep = sub(P[i], P[(i - 1 + nn) % nn]);
            const V2 en = sub(P[(i + 1) % nn], P[i]);
            ds[i] = 0.5 * (nrm(ep) + nrm(en));
            ang[i] = (mp.kappa_0 != 0.0) ? mp.kappa_0 * ds[i] : std::atan2(crs(ep, en), dt(ep, en));
        }
    }
}

// Capsule::centroid with minimum image in x (capsule.cpp:159-173).
V2 centroid_periodic(const std::vector<V2>& P, int nx) {
    const double Lx = static_cast<double>(nx);
    V2 ref = P[0], sum = ref;
    for (size_t i = 1; i < P.size(); ++i) {
        V2 d = sub(P[i], ref);
        if (nx > 0) {
            if (d.x > 0.5 * Lx) d.x -= Lx;
            if (d.x < -0.5 * Lx) d.x += Lx;
        }
        sum = {sum.x + (ref.x + d.x), sum.y + (ref.y + d.y)};
    }
    const double n = static_cast<double>(P.size());
    return {sum.x / n, sum.y / n};
}

}  // namespace

extern "C" int sfg_build_circle_capsule(double cx, double cy, double radius, int num_nodes,
                                        const sfg_membrane_params* mp,
                                        sfg_capsule_rest* rest_out, double* pos_out,
                                        double* rest_len_out, double* rest_ang_out,
                                        double* rest_ds_out, int capacity) {
    if (!mp || !rest_out) {
        sfg_host::set_error("sfg_build_circle_capsule: null argument");
        return SFG_ERR_ARG;
    }
    if (!(radius > 0.0)) {
        sfg_host::set_error("sfg_build_circle_capsule: radius must be positive");
        return SFG_ERR_ARG;
    }
    const int nn = num_nodes > 0 ? num_nodes : optimal_nodes(radius);
    rest_out->num_nodes = nn;
    if (!pos_out) return SFG_OK;  // size query
    if (nn > capacity) {
        sfg_host::set_error("sfg_build_circle_capsule: output capacity " +
                            std::to_string(capacity) + " < " + std::to_string(nn) + " nodes");
        return SFG_ERR_CAPACITY;
    }
    std::vector<V2> P;
    std::vector<double> L0, ang, ds;
    build_circle(cx, cy, radius, nn, *mp, *rest_out, P, L0, ang, ds);
    for (int i = 0; i < nn; ++i) {
        pos_out[2 * i] = P[i].x;
        pos_out[2 * i + 1] = P[i].y;
        if (rest_len_out) rest_len_out[i] = L0[i];
        if (rest_ang_out) rest_ang_out[i] = ang[i];
        if (rest_ds_out) rest_ds_out[i] = ds[i];
    }
    return SFG_OK;
}

// Simulation::addCapsuleRandom (simulation.cpp:220-274): the same engine and
// distributions, so the draws (x, y, r per attempt) are the reference's.
// Obstacle::signedDistance of CircleObstacle / RectObstacle
// (geometry/circle_obstacle.h:17-21, rect_obstacle.h:18-26); o = kind, a..d.
static double pillar_sd(const double* o, double x, double y) {
    if (o[0] == 0.0) {
        const double dx = x - o[1], dy = y - o[2];
        return std::sqrt(dx * dx + dy * dy) - o[3];
    }
    auto max3 = [](double a, double b, double c) {
        double m = a;
        if (m < b) m = b;
        if (m < c) m = c;
        return m;
    };
    const double dx = max3(o[1] - x, x - o[3], 0.0);
    const double dy = max3(o[2] - y, y - o[4], 0.0);
    const double outside = std::sqrt(dx * dx + dy * dy);
    if (outside > 1e-15) return outside;
    double m = x - o[1];
    if (o[3] - x < m) m = o[3] - x;
    if (y - o[2] < m) m = y - o[2];
    if (o[4] - y < m) m = o[4] - y;
    return -m;
}

extern "C" int sfg_place_random(int count, double x0, double y0, double x1, double y1,
                                double rmin, double rmax, int num_nodes, int seed, double min_gap,
                                int max_attempts, int check_walls, int nx, int ny, int n_existing,
                                const double* existing_centroid, const double* existing_radius,
                                int capacity, double* out_center, double* out_radius,
                                int* n_placed, int* n_attempts) {
    return sfg_place_random_pillars(count, x0, y0, x1, y1, rmin, rmax, num_nodes, seed, min_gap,
                                    max_attempts, check_walls, nx, ny, n_existing,
                                    existing_centroid, existing_radius, capacity, out_center,
                                    out_radius, n_placed, n_attempts, 0, nullptr);
}

extern "C" int sfg_place_random_pillars(int count, double x0, double y0, double x1, double y1,
                                        double rmin, double rmax, int num_nodes, int seed,
                                        double min_gap, int max_attempts, int check_walls, int nx,
                                        int ny, int n_existing, const double* existing_centroid,
                                        const double* existing_radius, int capacity,
                                        double* out_center, double* out_radius, int* n_placed,
                                        int* n_attempts, int n_pillars, const double* pillars) {
    if (n_pillars < 0 || (n_pillars > 0 && !pillars)) {
        sfg_host::set_error("sfg_place_random_pillars: bad pillar list");
        return SFG_ERR_ARG;
    }
    if (count < 0 || (n_existing > 0 && (!existing_centroid || !existing_radius))) {
        sfg_host::set_error("sfg_place_random: bad arguments");
        return SFG_ERR_ARG;
    }
    std::vector<V2> cen;
    std::vector<double> rad;
    for (int i = 0; i < n_existing; ++i) {
        cen.push_back({existing_centroid[2 * i], existing_centroid[2 * i + 1]});
        rad.push_back(existing_radius[i]);
    }
    std::mt19937 rng(static_cast<unsigned>(seed));
    std::uniform_real_distribution<double> dx(x0, x1), dy(y0, y1), dr(rmin, rmax);
    int placed = 0, attempts = 0;
    const int total_max = max_attempts > 0 ? max_attempts : count * 500;
    sfg_membrane_params mp{};
    while (placed < count && attempts < total_max) {
        const double cx = dx(rng);
        const double cy = dy(rng);
        const double r = dr(rng);
        bool overlap = false;
        for (size_t c = 0; c < cen.size(); ++c) {
            if (nrm(sub(V2{cx, cy}, cen[c])) < r + rad[c] + min_gap) {
                overlap = true;
                break;
            }
        }
        if (check_walls) {
            if (cy - r < 0.0 + min_gap || cy + r > static_cast<double>(ny - 1) - min_gap)
                overlap = true;
            // obstacles of the channel builder (simulation.cpp:256-261)
            for (int k = 0; k < n_pillars; ++k)
                if (pillar_sd(pillars + 5 * k, cx, cy) < r + min_gap) {
                    overlap = true;
                    break;
                }
        }
        if (!overlap) {
            if (placed >= capacity) {
                sfg_host::set_error("sfg_place_random: output capacity exceeded");
                return SFG_ERR_CAPACITY;
            }
            const int nn = num_nodes > 0 ? num_nodes : optimal_nodes(r);
            sfg_capsule_rest rest{};
            std::vector<V2> P;
            std::vector<double> L0, ang, ds;
            build_circle(cx, cy, r, nn, mp, rest, P, L0, ang, ds);
            cen.push_back(centroid_periodic(P, nx));
            rad.push_back(std::sqrt(rest.rest_area / kPi));
            out_center[2 * placed] = cx;
            out_center[2 * placed + 1] = cy;
            out_radius[placed] = r;
            ++placed;
        }
        ++attempts;
    }
    if (n_placed) *n_placed = placed;
    if (n_attempts) *n_attempts = attempts;
    return SFG_OK;
}
