// Output writer: the reference's field dumps (Files.cuh:73-211, called from cuOPO3D.cu:75-85)
// from one device-to-host copy per field.
//
// The reference's main writes, per field, NT text files of (x, y) slices and NX NY text
// files of time traces, each through its own full device-to-host copy of the field and
// an iostream at 20 significant digits: at 128 x 128 x 2048 that is 18,432 copies of the
// whole field and 37 k files.  Here one copy brings the field to the host and the files
// are formatted (std::to_chars, the same digits as "%.20g", which is what the reference's
// setprecision(20) stream prints) and written by a pool of host threads.  The binary form
// writes the whole field as one file instead.

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuopo3d.h"
#include "solver_internal.h"

namespace {

// Appends v as "%.20g" would print it.
inline void put20(std::string &out, double v)
{
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 20);
    out.append(buf, r.ptr);
}

bool write_file(const std::string &path, const std::string &data)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data.data(), 1, data.size(), f) == data.size();
    return std::fclose(f) == 0 && ok;
}

// Host copy of one field as (re, im) doubles in [t][y][x] order: FP32 values are widened
// exactly, so their printed digits are those of the float itself.
struct HostField {
    int nx = 0, ny = 0, nt = 0;
    std::vector<double> v;  // 2 per voxel
    double re(size_t i) const { return v[2 * i]; }
    double im(size_t i) const { return v[2 * i + 1]; }
};

// Runs job(k) for k in [0, n) on up to `threads` host threads; false if any job failed.
template <typename Job> bool parallel_jobs(size_t n, unsigned threads, Job job)
{
    std::atomic<size_t> next{0};
    std::atomic<bool> ok{true};
    auto worker = [&] {
        for (size_t k; (k = next.fetch_add(1)) < n && ok.load();)
            if (!job(k)) ok.store(false);
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < threads; t++) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
    return ok.load();
}

}  // namespace

extern "C" int opo_save_fields(OpoSolver *s, int which, const char *slice_prefix, const char *trace_prefix,
                               int format)
{
    if (!s || which < 0 || which > 3 || (format != OPO_FILES_TEXT && format != OPO_FILES_BINARY) ||
        (!slice_prefix && !trace_prefix) || (format == OPO_FILES_BINARY && !slice_prefix))
        return OPO_ERR_INVALID;
    const OpoParams &p = opo::solver_params(s);
    HostField h;
    h.nx = p.nx;
    h.ny = p.ny;
    h.nt = p.nt;
    const size_t V = (size_t)p.nx * p.ny * p.nt;
    const bool fp64 = p.precision == OPO_FP64;
    // one device-to-host copy of the field in its own precision (the call waits for it)
    std::vector<float> f32;
    h.v.resize(2 * V);
    int rc;
    if (fp64) {
        rc = opo_get_field(s, which, h.v.data(), OPO_MEM_HOST, OPO_FP64);
    } else {
        f32.resize(2 * V);
        rc = opo_get_field(s, which, f32.data(), OPO_MEM_HOST, OPO_FP32);
    }
    if (rc) return rc;
    if (format == OPO_FILES_BINARY) {
        // header (32 bytes): "OPO3DFLD", version 1, nx, ny, nt, bytes per complex value,
        // field index; then the field, [t][y][x], in the solver's precision
        std::string data(32, '\0');
        const int hdr[6] = {1, p.nx, p.ny, p.nt, fp64 ? 16 : 8, which};
        std::memcpy(&data[0], "OPO3DFLD", 8);
        std::memcpy(&data[8], hdr, sizeof(hdr));
        const char *src = fp64 ? reinterpret_cast<const char *>(h.v.data()) : reinterpret_cast<const char *>(f32.data());
        data.append(src, (fp64 ? 16 : 8) * V);
        return write_file(std::string(slice_prefix) + ".bin", data) ? OPO_OK : OPO_ERR_INVALID;
    }
    if (!fp64)
        for (size_t k = 0; k < 2 * V; k++) h.v[k] = (double)f32[k];
    const unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t plane = (size_t)p.nx * p.ny;
    // (x, y) slice t: NY rows of NX values, each followed by a tab (Files.cuh:73-94)
    auto slice_job = [&](size_t t) {
        const std::string base = std::string(slice_prefix) + std::to_string(t);
        for (int part = 0; part < 2; part++) {
            std::string out;
            out.reserve(plane * 26 + (size_t)p.ny);
            for (int y = 0; y < p.ny; y++) {
                for (int x = 0; x < p.nx; x++) {
                    const size_t i = t * plane + (size_t)y * p.nx + x;
                    put20(out, part ? h.im(i) : h.re(i));
                    out += '\t';
                }
                out += '\n';
            }
            if (!write_file(base + (part ? "_i.dat" : "_r.dat"), out)) return false;
        }
        return true;
    };
    // time trace of pixel (x, y): NT values, one per line (Files.cuh:178-194); pixel
    // k = x NY + y, the reference main's loop order (cuOPO3D.cu:82-86)
    auto trace_job = [&](size_t k) {
        const int x = (int)(k / p.ny), y = (int)(k % p.ny);
        const std::string base = std::string(trace_prefix) + std::to_string(x) + "_y_" + std::to_string(y);
        for (int part = 0; part < 2; part++) {
            std::string out;
            out.reserve((size_t)p.nt * 26);
            for (int t = 0; t < p.nt; t++) {
                const size_t i = (size_t)t * plane + (size_t)y * p.nx + x;
                put20(out, part ? h.im(i) : h.re(i));
                out += '\n';
            }
            if (!write_file(base + (part ? "_i.dat" : "_r.dat"), out)) return false;
        }
        return true;
    };
    if (slice_prefix && !parallel_jobs((size_t)p.nt, threads, slice_job)) return OPO_ERR_INVALID;
    if (trace_prefix && !parallel_jobs(plane, threads, trace_job)) return OPO_ERR_INVALID;
    return OPO_OK;
}
