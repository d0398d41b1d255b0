// Utilities the cuOPO3D programs call: error check, timers, status lines, indexing.
#pragma once

#include "DtypesConsts.cuh"

#define CHECK(call)                                                                        \
    {                                                                                      \
        const cudaError_t err_ = (call);                                                   \
        if (err_ != cudaSuccess) {                                                         \
            fprintf(stderr, "Error: %s:%d, code: %d, reason: %s\n", __FILE__, __LINE__,    \
                    (int)err_, cudaGetErrorString(err_));                                  \
            exit(1);                                                                       \
        }                                                                                  \
    }

inline void printLineOnScreen() { std::cout << std::string(67, '-') << std::endl; }

inline double seconds()
{
    static const auto start = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

inline void TimingCode(double s)
{
    if (s < 60.) std::cout << "\n\nTime elapsed " << s << " seconds\n" << std::endl;
    else if (s < 3600.) std::cout << "\n\nTime elapsed " << s / 60 << " minutes\n" << std::endl;
    else std::cout << "\n\nTime elapsed " << s / 3600 << " hours\n" << std::endl;
}

inline real_t measuredTime(real_t tic) { return (real_t)(seconds() - tic); }

inline void runOPO_status(uint32_t r, uint32_t every)
{
    if (every && r != 0 && (r % every == 0 || r == NRT - 1))
        std::cout << "# Round trip: " << r << " - Completed " << r * 100 / NRT << "%" << std::endl;
}

// Element (x, y, t) of a field stored [t][y][x].
__host__ __device__ inline uint32_t IDX(uint32_t x, uint32_t y, uint32_t t) { return t * (NX * NY) + y * NX + x; }

template <typename T> void linspace(T &v, real_t xmin, real_t xmax)
{
    for (uint32_t i = 0; i < v.size(); i++) v[i] = xmin + i * (xmax - xmin) / (v.size() - 1);
}

inline void is_gpu_available()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        std::cerr << "No CUDA device available." << std::endl;
        exit(1);
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    printLineOnScreen();
    std::cout << "\n\nUsing Device " << dev << ": GPU " << prop.name << "\n" << std::endl;
}

inline void printGrid()
{
    printLineOnScreen();
    std::cout << "\nSpatio-temporal grid:\n        ---> (NT, NX, NY, NZ) = (" << NT << ", " << NX << ", " << NY
              << ", " << NZ << ")\n        ---> SIZE = NT*NX*NY = " << SIZE << "\n" << std::endl;
}

namespace opo_files {
// Generation of the drop-in's device fields, for the savers' host snapshots (Files.cuh):
// bumped by every drop-in member that writes a field (Solver runs, EFields' pump and noise
// setters, Cavity::applyReflectivity).  Code that writes a field directly between two saves
// of it calls opo_files::invalidate() so that the next save copies it again.
inline unsigned long long &generation()
{
    static unsigned long long g = 0;
    return g;
}
inline void invalidate() { generation()++; }
}  // namespace opo_files
