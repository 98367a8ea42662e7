// crysscft_b200_solvers.hpp — CrysPSSolverBase adapters over the C ABI.
//
// Include AFTER the reference's "solver_base.h" (class CrysPSSolverBase,
// src/solver_base.h:8-51).  The three classes are drop-ins for CrysPSSolverP1
// (src/solver_p1.h:14-53), CrysPSSolver3m (src/solver_3m.h:14-53) and
// CrysPSSolverPmmm (src/solver_Pmmm.h:13-53): same constructor arguments, same
// virtuals, and get_iomat_for_diffusion() returns a host buffer that diffusion()
// transforms in place, so the reference's solve_diffusion_equation and
// diblock_scft_simple_iterate (src/crysSCFT_sample.cpp:373-531) run on the GPU
// without changes.  Like the reference, an error prints "ERROR ..." and exits.
#pragma once

#include <cstdlib>
#include <iostream>

#include "crysscft_b200.h"

namespace crysscft_b200 {

class GpuSolverAdapter : public CrysPSSolverBase {
public:
    GpuSolverAdapter(int kind, const c_array<size_t, 3>& grid_size_log, const double* translational_part = nullptr)
        : CrysPSSolverBase(grid_size_log) {
        const size_t g[3] = {grid_size_log[0], grid_size_log[1], grid_size_log[2]};
        check(scft_solver_create(kind, g, translational_part, SCFT_FP64, -1, &h_));
        size_t phy[3];
        check(scft_solver_get_grid_size_phy(h_, phy));
        grid_size_phy_ = {phy[0], phy[1], phy[2]};
        space_size_phy_ = phy[0] * phy[1] * phy[2];
        check(scft_solver_get_iomat_for_diffusion(h_, &iomat_for_diffusion_));
    }
    ~GpuSolverAdapter() override { scft_solver_destroy(h_); }

    void set_cell_para(const c_array<double, 6>& cell_para) override {
        check(scft_solver_set_cell_para(h_, cell_para.arr));
        double c[6];
        check(scft_solver_get_cell_para(h_, c));
        cell_para_ = {c[0], c[1], c[2], c[3], c[4], c[5]};
        ds_current_ = 0.00;
    }
    void set_contour_step(double ds) override {
        check(scft_solver_set_contour_step(h_, ds));
        ds_current_ = ds;
    }
    void diffusion() const override { check(scft_solver_diffusion(h_)); }

    scft_solver_t handle() const { return h_; }

private:
    static void check(int status) {
        if (status != SCFT_OK) {
            std::cout << "ERROR: " << scft_status_string(status) << ": " << scft_last_error() << std::endl;
            exit(1);
        }
    }
    scft_solver_t h_ = nullptr;
};

class CrysPSSolverP1Gpu : public GpuSolverAdapter {
public:
    explicit CrysPSSolverP1Gpu(const c_array<size_t, 3>& grid_size_log)
        : GpuSolverAdapter(SCFT_SOLVER_P1, grid_size_log) {}
};

class CrysPSSolver3mGpu : public GpuSolverAdapter {
public:
    CrysPSSolver3mGpu(const c_array<size_t, 3>& grid_size_log,
                      const c_array<double, 9> translational_part = {0, 0, 0, 0, 0, 0, 0, 0, 0})
        : GpuSolverAdapter(SCFT_SOLVER_3M, grid_size_log, translational_part.arr) {}
};

class CrysPSSolverPmmmGpu : public GpuSolverAdapter {
public:
    explicit CrysPSSolverPmmmGpu(const c_array<size_t, 3>& grid_size_log)
        : GpuSolverAdapter(SCFT_SOLVER_PMMM, grid_size_log) {}
};

}  // namespace crysscft_b200
