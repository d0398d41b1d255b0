// Text writers with the file names and format of cuOPO3D's savers (20 significant
// digits, "_r.dat" / "_i.dat" pairs).  The device overloads read a host snapshot of the
// field, taken with one device-to-host copy and reused by every later save of the same
// field while no drop-in member has written the fields since (main's loops over NT slices
// and NX NY pixels then cost one copy per field, not one per file).  Numbers are formatted
// with std::to_chars to the digits of "%.20g", which is what the reference's
// setprecision(20) streams print.
#pragma once

#include <charconv>

#include "Common.cuh"

namespace opo_files {
struct Snapshot {
    const void *ptr = nullptr;
    size_t n = 0;
    unsigned long long gen = ~0ull;
    std::vector<complex_t> h;
};
// Host copy of device field V (the four most recent fields are kept).
inline const std::vector<complex_t> &snapshot(const cVecd_t &V)
{
    static Snapshot cache[4];
    static unsigned next = 0;
    const void *p = thrust::raw_pointer_cast(V.data());
    for (auto &c : cache)
        if (c.ptr == p && c.n == V.size() && c.gen == generation()) return c.h;
    Snapshot &c = cache[next++ % 4];
    c.ptr = p;
    c.n = V.size();
    c.gen = generation();
    c.h.resize(V.size());
    CHECK(cudaMemcpy(c.h.data(), p, sizeof(complex_t) * V.size(), cudaMemcpyDeviceToHost));
    return c.h;
}

inline void put20(std::string &out, double v)
{
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 20);
    out.append(buf, r.ptr);
}
inline void write_text(const std::string &name, const std::string &s)
{
    std::ofstream f(name, std::ios::binary);
    f << s;
}
inline void write_column(const std::string &name, const std::vector<double> &v)
{
    std::string s;
    for (double x : v) {
        put20(s, x);
        s += '\n';
    }
    write_text(name, s);
}
inline void write_pair(const std::string &name, const std::vector<complex_t> &v)
{
    std::vector<double> re(v.size()), im(v.size());
    for (size_t k = 0; k < v.size(); k++) { re[k] = v[k].x; im[k] = v[k].y; }
    write_column(name + "_r.dat", re);
    write_column(name + "_i.dat", im);
}
// (x, y) slice `slice` of field m (NX NY NT values or one NX NY plane with slice 0)
inline void write_matrix(const std::string &name, const complex_t *m)
{
    for (int part = 0; part < 2; part++) {
        std::string s;
        for (uint32_t iy = 0; iy < NY; iy++) {
            for (uint32_t ix = 0; ix < NX; ix++) {
                put20(s, part ? m[iy * NX + ix].y : m[iy * NX + ix].x);
                s += '\t';
            }
            s += '\n';
        }
        write_text(name + (part ? "_i.dat" : "_r.dat"), s);
    }
}
inline std::vector<complex_t> trace(const complex_t *V, uint32_t x, uint32_t y)
{
    std::vector<complex_t> tr(NT);
    for (uint32_t t = 0; t < NT; t++) tr[t] = V[IDX(x, y, t)];
    return tr;
}
}  // namespace opo_files

inline void SaveVectorReal(const rVech_t &V, std::string name)
{
    opo_files::write_column(name + ".dat", std::vector<double>(V.begin(), V.end()));
}
inline void SaveVectorRealGPU(const rVecd_t &V, std::string name) { SaveVectorReal(rVech_t(V), name); }
inline void SaveVectorComplex(const cVech_t &V, std::string name)
{
    opo_files::write_pair(name, std::vector<complex_t>(V.begin(), V.end()));
}
inline void SaveVectorComplexGPU(const cVecd_t &V, std::string name) { SaveVectorComplex(cVech_t(V), name); }

inline void saveMatrixComplex_TimeSlice(const cVech_t &V, uint32_t slice, std::string name)
{
    opo_files::write_matrix(name, thrust::raw_pointer_cast(V.data()) + (size_t)slice * NX * NY);
}
inline void saveMatrixComplex_TimeSlice(const cVecd_t &V, uint32_t slice, std::string name)
{
    opo_files::write_matrix(name, opo_files::snapshot(V).data() + (size_t)slice * NX * NY);
}
inline void saveMatrixComplex_TimeSlice_GPU(const cVecd_t &V, uint32_t slice, std::string name)
{
    saveMatrixComplex_TimeSlice(V, slice, name);
}
inline void saveMatrixComplex(const cVech_t &M, std::string name) { saveMatrixComplex_TimeSlice(M, 0, name); }
inline void saveMatrixComplexGPU(const cVecd_t &M, std::string name) { saveMatrixComplex_TimeSlice(M, 0, name); }

inline void SaveElectricField1D_time(const cVech_t &V, std::string name)
{
    opo_files::write_pair(name, std::vector<complex_t>(V.begin(), V.begin() + NT));
}
inline void SaveElectricField1D_time_GPU(const cVecd_t &V, std::string name) { SaveElectricField1D_time(cVech_t(V), name); }

inline void SaveElectricField3D_time(const cVech_t &V, uint32_t x, uint32_t y, std::string name)
{
    opo_files::write_pair(name, opo_files::trace(thrust::raw_pointer_cast(V.data()), x, y));
}
inline void SaveElectricField_time3D_GPU(const cVecd_t &V, uint32_t x, uint32_t y, std::string name)
{
    opo_files::write_pair(name, opo_files::trace(opo_files::snapshot(V).data(), x, y));
}

inline void saveAppendedValues2Columns(std::string name, real_t a, real_t b)
{
    std::ofstream f(name + ".txt", std::ios::app);
    if (f.is_open()) f << a << "\t" << b << std::endl;
    else std::cerr << "Unable to open the file for writing." << std::endl;
}
