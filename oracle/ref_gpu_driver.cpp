// The reference's own driver on the GPU solvers — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's src/crysSCFT_sample.cpp unmodified (main renamed, as in
// ref_harness.cpp) together with the CrysPSSolverBase adapters of
// include/crysscft_b200_solvers.hpp, so the reference's diblock_scft_simple_iterate
// and solve_diffusion_equation (src/crysSCFT_sample.cpp:373-531) drive the B200
// library through the plug-in interface exactly as they drive the CPU solvers.
// Built by `make -C oracle gpu_driver` into oracle/_ref/libref_gpu_driver.so.
#include <mm_malloc.h>
#define main crysscft_reference_main
#include "crysSCFT_sample.cpp"
#undef main

#include <cstring>
#include <memory>
#include <sstream>

#include "crysscft_b200_solvers.hpp"

extern "C" long refgpu_run_driver(int kind, long nx, long ny, long nz, double fA, double ds, double xN, double Lx,
                                  double Ly, double Lz, double acceptance, long Nstep, const double* wA0,
                                  const double* wB0, const char* name, char* log, long logcap) {
    c_array<size_t, 3> grid = {{(size_t)nx, (size_t)ny, (size_t)nz}};
    std::unique_ptr<CrysPSSolverBase> solver;
    if (kind == 0) solver.reset(new crysscft_b200::CrysPSSolverP1Gpu(grid));
    else if (kind == 1) solver.reset(new crysscft_b200::CrysPSSolver3mGpu(grid));
    else solver.reset(new crysscft_b200::CrysPSSolverPmmmGpu(grid));
    const size_t size = solver->get_space_size_phy();
    auto init = [size, wA0, wB0](double* wA, double* wB) -> void {
        for (size_t itr = 0; itr < size; ++itr) {
            wA[itr] = wA0[itr];
            wB[itr] = wB0[itr];
        }
    };
    std::ostringstream cap;
    std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
    std::clock_t t = diblock_scft_simple_iterate((size_t)nx, (size_t)ny, (size_t)nz, fA, ds, xN, Lx, Ly, Lz,
                                                 acceptance, (size_t)Nstep, std::string(name), *solver, init);
    std::cout.rdbuf(old);
    const std::string s = cap.str();
    if (log && logcap > 0) {
        const size_t n = s.size() < (size_t)(logcap - 1) ? s.size() : (size_t)(logcap - 1);
        std::memcpy(log, s.data(), n);
        log[n] = 0;
    }
    return (long)t;
}
