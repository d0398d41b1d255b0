// Text writers with the file names and format of cuOPO3D's savers (20 significant
// digits, "_r.dat" / "_i.dat" pairs).  The device overloads copy only the part a file
// holds -- one t-slice (contiguous) or one pixel's time trace (strided) -- instead of
// the whole field for every file.
#pragma once

#include "Common.cuh"

namespace opo_files {
inline void write_column(const std::string &name, const std::vector<double> &v)
{
    std::ofstream f(name);
    for (double x : v) f << std::setprecision(20) << x << "\n";
}
inline void write_pair(const std::string &name, const std::vector<complex_t> &v)
{
    std::vector<double> re(v.size()), im(v.size());
    for (size_t k = 0; k < v.size(); k++) { re[k] = v[k].x; im[k] = v[k].y; }
    write_column(name + "_r.dat", re);
    write_column(name + "_i.dat", im);
}
inline void write_matrix(const std::string &name, const std::vector<complex_t> &m)
{
    for (int part = 0; part < 2; part++) {
        std::ofstream f(name + (part ? "_i.dat" : "_r.dat"));
        for (uint32_t iy = 0; iy < NY; iy++) {
            for (uint32_t ix = 0; ix < NX; ix++)
                f << std::setprecision(20) << (part ? m[iy * NX + ix].y : m[iy * NX + ix].x) << "\t";
            f << "\n";
        }
    }
}
inline std::vector<complex_t> device_slice(const cVecd_t &V, uint32_t slice)
{
    std::vector<complex_t> h(NX * NY);
    CHECK(cudaMemcpy(h.data(), thrust::raw_pointer_cast(V.data()) + (size_t)slice * NX * NY,
                     sizeof(complex_t) * NX * NY, cudaMemcpyDeviceToHost));
    return h;
}
inline std::vector<complex_t> device_trace(const cVecd_t &V, uint32_t x, uint32_t y)
{
    std::vector<complex_t> h(NT);
    CHECK(cudaMemcpy2D(h.data(), sizeof(complex_t), thrust::raw_pointer_cast(V.data()) + (size_t)y * NX + x,
                       sizeof(complex_t) * NX * NY, sizeof(complex_t), NT, cudaMemcpyDeviceToHost));
    return h;
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
    opo_files::write_matrix(name, std::vector<complex_t>(V.begin() + (size_t)slice * NX * NY,
                                                         V.begin() + (size_t)(slice + 1) * NX * NY));
}
inline void saveMatrixComplex_TimeSlice(const cVecd_t &V, uint32_t slice, std::string name)
{
    opo_files::write_matrix(name, opo_files::device_slice(V, slice));
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
    std::vector<complex_t> tr(NT);
    for (uint32_t t = 0; t < NT; t++) tr[t] = V[IDX(x, y, t)];
    opo_files::write_pair(name, tr);
}
inline void SaveElectricField_time3D_GPU(const cVecd_t &V, uint32_t x, uint32_t y, std::string name)
{
    opo_files::write_pair(name, opo_files::device_trace(V, x, y));
}

inline void saveAppendedValues2Columns(std::string name, real_t a, real_t b)
{
    std::ofstream f(name + ".txt", std::ios::app);
    if (f.is_open()) f << a << "\t" << b << std::endl;
    else std::cerr << "Unable to open the file for writing." << std::endl;
}
