// Threshold sweeps: the reference's main use case, a (pump power, waist) scan that runs
// one OPO per point and records its output power (cuOPO3D.sh:58-80 re-runs the binary
// per point; cuOPO3D.cu:88 appends power pairs with saveAppendedValues2Columns,
// Files.cuh:215-233), run here as waves of instances on one OpoBatch.
//
// Every point advances by whole round trips with FP64 tallies of its fields after each
// one (opo_batch_sums); a point whose fields stop being finite leaves the batch at once
// (the reference's NaN probe, Solver3D.cuh:999-1005).  After the run, the signal's
// round-trip gain over the last `window` round trips, g = (Ps(n) / Ps(n - window))^(1 /
// window), says whether the point is above threshold (g > 1: the signal grows) or below
// (g < 1: cavity losses win).  opo_sweep_threshold brackets the threshold pump power from
// those gains and interpolates ln g to zero between the bracketing points.

#include <algorithm>
#include <cmath>
#include <fstream>
#include <limits>
#include <vector>

#include "../../include/cuopo3d.h"

extern "C" int opo_sweep(const OpoConfig *base, OpoSweepPoint *pts, int n, const OpoSweepOptions *opt,
                         double *tallies)
{
    if (!base || !pts || n < 0 || !opt || opt->round_trips < 1 || opt->window < 1 ||
        opt->window > opt->round_trips)
        return OPO_ERR_INVALID;
    const int R = opt->round_trips;
    const int cap = std::max(1, std::min(n, opt->capacity > 0 ? opt->capacity : n));
    OpoBatch *b = nullptr;
    int rc = opo_batch_create(opt->precision, cap, opt->hbm_budget, opt->tuning_set ? opt->tuning : nullptr, &b);
    if (rc) return rc;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (tallies)
        for (size_t k = 0; k < (size_t)n * R * 3; k++) tallies[k] = nan;
    for (int k = 0; k < n; k++) {
        pts[k].status = -1;
        pts[k].round_trips = 0;
        for (int f = 0; f < 3; f++) pts[k].sums[f] = pts[k].power_xy[f] = nan;
        pts[k].output_power = pts[k].gain = nan;
        pts[k].above = 0;
    }
    std::vector<double> sums(3 * (size_t)cap), ps((size_t)n * (R + 1), nan);
    auto cfg_of = [&](int k) {
        OpoConfig c = *base;
        c.P = pts[k].P;
        c.w0 = pts[k].w0;
        c.total_rt = R;
        c.precision = opt->precision;
        return c;
    };
    int next = 0;
    while (next < n) {
        // admit the next wave: as many points as fit the slots and the budget
        std::vector<std::pair<int, int>> live;  // (point, slot)
        while (next < n) {
            OpoConfig c = cfg_of(next);
            OpoParams p;
            if (opo_params_from_config(&c, &p, nullptr) != OPO_OK) {
                pts[next++].status = OPO_ERR_INVALID;
                continue;
            }
            std::vector<double> w(p.nt);
            opo_time_freq(p.nt, p.t_window, nullptr, w.data());
            int slot = -1;
            rc = opo_batch_add(b, &p, w.data(), &slot);
            if (rc == OPO_ERR_CAPACITY && !live.empty()) break;  // run this wave first
            if (rc) {
                pts[next++].status = rc;  // does not fit even alone, or not supported
                continue;
            }
            if ((rc = opo_batch_init_fields(b, slot, &c, opt->seed + (uint64_t)next, opt->noise_sigma, 0))) {
                opo_batch_destroy(b);
                return rc;
            }
            live.emplace_back(next++, slot);
        }
        if (live.empty()) continue;
        // tallies of the initial fields (round trip 0), for windows that start there
        if ((rc = opo_batch_sums(b, sums.data()))) {
            opo_batch_destroy(b);
            return rc;
        }
        for (auto &L : live) ps[(size_t)L.first * (R + 1)] = sums[3 * (size_t)L.second + 1];
        for (int r = 1; r <= R && !live.empty(); r++) {
            if ((rc = opo_batch_run_round_trips(b, 1)) || (rc = opo_batch_sums(b, sums.data()))) {
                opo_batch_destroy(b);
                return rc;
            }
            for (size_t j = 0; j < live.size();) {
                const int k = live[j].first, slot = live[j].second;
                const double *sk = &sums[3 * (size_t)slot];
                pts[k].round_trips = r;
                ps[(size_t)k * (R + 1) + r] = sk[1];
                if (tallies)
                    for (int f = 0; f < 3; f++) tallies[((size_t)k * R + (r - 1)) * 3 + f] = sk[f];
                const bool finite = std::isfinite(sk[0]) && std::isfinite(sk[1]) && std::isfinite(sk[2]);
                if (!finite || r == R) {
                    pts[k].status = finite ? OPO_OK : OPO_ERR_NONFINITE;
                    for (int f = 0; f < 3; f++) pts[k].sums[f] = sk[f];
                    OpoConfig c = cfg_of(k);
                    if (opo_power_cut_xy(&c, sk, pts[k].power_xy) == OPO_OK)
                        pts[k].output_power = pts[k].power_xy[1] * (1.0 - c.Rs);
                    const double a = ps[(size_t)k * (R + 1) + r - opt->window], z = ps[(size_t)k * (R + 1) + r];
                    if (finite && r == R && a > 0 && z >= 0) {
                        pts[k].gain = std::pow(z / a, 1.0 / opt->window);
                        pts[k].above = pts[k].gain > 1.0 ? 1 : 0;
                    }
                    opo_batch_remove(b, slot);
                    live.erase(live.begin() + (long)j);
                } else {
                    j++;
                }
            }
        }
    }
    opo_batch_destroy(b);
    return OPO_OK;
}

extern "C" int opo_sweep_threshold(const OpoSweepPoint *pts, int n, double *p_below, double *p_above,
                                   double *p_est)
{
    if (!pts || n < 0 || !p_below || !p_above || !p_est) return OPO_ERR_INVALID;
    // largest power below threshold that is under the smallest power above it
    double above = std::numeric_limits<double>::infinity();
    int ia = -1;
    for (int k = 0; k < n; k++)
        if (pts[k].status == OPO_OK && std::isfinite(pts[k].gain) && pts[k].above && pts[k].P < above) {
            above = pts[k].P;
            ia = k;
        }
    double below = -std::numeric_limits<double>::infinity();
    int ib = -1;
    for (int k = 0; k < n; k++)
        if (pts[k].status == OPO_OK && std::isfinite(pts[k].gain) && !pts[k].above && pts[k].P < above &&
            pts[k].P > below) {
            below = pts[k].P;
            ib = k;
        }
    if (ia < 0 || ib < 0) return OPO_ERR_INVALID;  // no crossing in the scanned range
    *p_below = below;
    *p_above = above;
    // ln g is ~linear in the pump power near threshold (small-signal gain ~ P)
    const double la = std::log(pts[ia].gain), lb = std::log(pts[ib].gain);
    *p_est = la > lb ? below + (above - below) * (0.0 - lb) / (la - lb) : 0.5 * (below + above);
    return OPO_OK;
}

extern "C" int opo_sweep_write(const char *path, const OpoSweepPoint *pts, int n, int append)
{
    if (!path || !pts || n < 0) return OPO_ERR_INVALID;
    // saveAppendedValues2Columns (Files.cuh:218-233): "value1 \t value2" per line with the
    // stream's default formatting; here pump power and output-coupled signal power
    std::ofstream f(path, append ? std::ios::app : std::ios::trunc);
    if (!f.is_open()) return OPO_ERR_INVALID;
    for (int k = 0; k < n; k++)
        if (pts[k].status == OPO_OK) f << pts[k].P << "\t" << pts[k].output_power << std::endl;
    return f.good() ? OPO_OK : OPO_ERR_INVALID;
}
