// Reference harness — TEST INFRASTRUCTURE ONLY (oracle).  Not part of the product.
//
// Compiles the reference program's own translation unit, src/crysSCFT_sample.cpp,
// unmodified and from where it lies (the recipe in oracle/Makefile passes the
// reference's src directory on the include path), together with the FFTW-API
// shim in oracle/fftw_shim (FFTW 3.3.3 is not installed on this machine).
// `main` is renamed so the file can be linked as a library; nothing else in the
// reference is touched.  The extern "C" functions below only forward to the
// reference's classes and free functions so tests and the CPU baseline can
// drive them through ctypes:
//
//   solvers     CrysPSSolverP1 / CrysPSSolver3m / CrysPSSolverPmmm
//               (src/solver_p1.h, src/solver_3m.h, src/solver_Pmmm.h)
//   contour     solve_diffusion_equation      src/crysSCFT_sample.cpp:373-396
//   helpers     array_exp / calc_ksi / integrate_phi / calc_new_fields /
//               array_average                 src/crysSCFT_sample.cpp:294-371
//   driver      diblock_scft_simple_iterate   src/crysSCFT_sample.cpp:426-531
//
// ref_scft_run repeats the driver's loop body (src/crysSCFT_sample.cpp:476-508)
// statement for statement with the reference's own helper functions, and
// evaluates the free-energy terms of print_energy (src/crysSCFT_sample.cpp:398-424)
// at full precision every iteration (print_energy itself only prints 10 digits).
// ref_run_driver runs the unmodified template driver and returns what it prints,
// which pins ref_scft_run to the reference's own loop.

#include <mm_malloc.h>
#define main crysscft_reference_main
#include "crysSCFT_sample.cpp"
#undef main

#include <chrono>
#include <cstring>
#include <memory>
#include <sstream>

namespace {

enum { REF_P1 = 0, REF_3M = 1, REF_PMMM = 2 };

struct RefSolver {
    std::unique_ptr<CrysPSSolverBase> s;
};

CrysPSSolverBase* make_solver(int kind, long nx, long ny, long nz, const double* g9) {
    c_array<size_t, 3> grid = {{(size_t)nx, (size_t)ny, (size_t)nz}};
    if (kind == REF_P1) return new CrysPSSolverP1(grid);
    if (kind == REF_3M) {
        c_array<double, 9> g = {{0, 0, 0, 0, 0, 0, 0, 0, 0}};
        if (g9)
            for (int i = 0; i < 9; ++i) g.arr[i] = g9[i];
        return new CrysPSSolver3m(grid, g);
    }
    return new CrysPSSolverPmmm(grid);
}

// free-energy terms exactly as print_energy (src/crysSCFT_sample.cpp:398-424) forms them
void energy_terms(double Q, double xN, const double* wA, const double* wB, const double* phiA,
                  const double* phiB, const double* ksi, size_t size, double* parts,
                  double* maxinc_out) {
    double fe_entropic_0 = -std::log(Q);
    double fe_entropic_1 = 0;
    double fe_enthalpic = 0;
    double fe_ksi = 0;
    double maxincomp = std::fabs(1 - phiA[0] - phiB[0]);
    for (size_t itr = 0; itr < size; ++itr) {
        fe_entropic_1 += -wA[itr] * phiA[itr] - wB[itr] * phiB[itr];
        fe_enthalpic += xN * phiA[itr] * phiB[itr];
        double temp = 1 - phiA[itr] - phiB[itr];
        fe_ksi += -ksi[itr] * temp;
        maxincomp = std::fabs(temp) > maxincomp ? std::fabs(temp) : maxincomp;
    }
    fe_entropic_1 /= size;
    fe_enthalpic /= size;
    fe_ksi /= size;
    parts[0] = fe_enthalpic;
    parts[1] = fe_entropic_0;
    parts[2] = fe_entropic_1;
    parts[3] = fe_ksi;
    *maxinc_out = maxincomp;
}

}  // namespace

extern "C" {

void* ref_solver_create(int kind, long nx, long ny, long nz, const double* g9) {
    auto* r = new RefSolver;
    r->s.reset(make_solver(kind, nx, ny, nz, g9));
    return r;
}

void ref_solver_destroy(void* h) { delete static_cast<RefSolver*>(h); }

void ref_solver_set_cell_para(void* h, const double* cell6) {
    c_array<double, 6> c = {{cell6[0], cell6[1], cell6[2], cell6[3], cell6[4], cell6[5]}};
    static_cast<RefSolver*>(h)->s->set_cell_para(c);
}

void ref_solver_set_contour_step(void* h, double ds) {
    static_cast<RefSolver*>(h)->s->set_contour_step(ds);
}

long ref_solver_space_size_phy(void* h) {
    return (long)static_cast<RefSolver*>(h)->s->get_space_size_phy();
}

void ref_solver_grid_size_phy(void* h, long* out3) {
    auto g = static_cast<RefSolver*>(h)->s->get_grid_size_phy();
    for (int i = 0; i < 3; ++i) out3[i] = (long)g[i];
}

// one triplet on a caller buffer: copy in -> CrysPSSolverBase::diffusion() -> copy out
void ref_solver_diffusion(void* h, double* io) {
    CrysPSSolverBase* s = static_cast<RefSolver*>(h)->s.get();
    size_t n = s->get_space_size_phy();
    double* iomat = s->get_iomat_for_diffusion();
    std::memcpy(iomat, io, n * sizeof(double));
    s->diffusion();
    std::memcpy(io, iomat, n * sizeof(double));
}

// solve_diffusion_equation (src/crysSCFT_sample.cpp:373-396) through the reference itself
double ref_solve_diffusion_equation(void* h, double* q, const double* init, const double* wds,
                                    long Ns, int direction) {
    std::clock_t t = 0;
    solve_diffusion_equation(q, init, wds, *static_cast<RefSolver*>(h)->s, (size_t)Ns, direction, t);
    return (double)t / CLOCKS_PER_SEC;
}

void ref_array_exp(double* dst, const double* src, double coef, double index, long size) {
    array_exp(dst, src, coef, index, (size_t)size);
}
void ref_calc_ksi(double* ksi, const double* wA, const double* wB, long size, double xN) {
    calc_ksi(ksi, wA, wB, (size_t)size, xN);
}
void ref_integrate_phi(double* phi, const double* q, const double* qc, double f, double Q,
                       long size, long Ns) {
    integrate_phi(phi, q, qc, f, Q, (size_t)size, (size_t)Ns);
}
void ref_calc_new_fields(double* wA, double* wB, const double* phiA, const double* phiB,
                         const double* ksi, double xN, double acc, long size) {
    calc_new_fields(wA, wB, phiA, phiB, ksi, xN, acc, (size_t)size);
}
double ref_array_average(const double* src, long size) { return array_average(src, (size_t)size); }

void ref_energy_terms(double Q, double xN, const double* wA, const double* wB, const double* phiA,
                      const double* phiB, const double* ksi, long size, double* parts4,
                      double* maxinc) {
    energy_terms(Q, xN, wA, wB, phiA, phiB, ksi, (size_t)size, parts4, maxinc);
}

// The loop of diblock_scft_simple_iterate (src/crysSCFT_sample.cpp:440-508), with the
// solver handle created by the caller and the initial fields passed in.  Outputs per
// iteration: F, the four energy parts, max incompressibility and Q.  Final phiA, phiB
// and the fields after the last update are written back.  Returns the wall time of
// the iteration loop in seconds (std::chrono::steady_clock); *triplet_cpu_seconds gets
// the reference's own std::clock() sum over diffusion() calls.
double ref_scft_run(void* h, double fA, double ds, double xN, double Lx, double Ly, double Lz,
                    double acceptance, long Nstep, const double* wA0, const double* wB0,
                    double* F_out, double* parts_out, double* maxinc_out, double* Q_out,
                    double* phiA_out, double* phiB_out, double* wA_out, double* wB_out,
                    double* triplet_cpu_seconds) {
    CrysPSSolverBase& solver = *static_cast<RefSolver*>(h)->s;
    constexpr size_t alignment = Alignment::value;
    size_t size = solver.get_space_size_phy();
    double fB = 1 - fA;
    size_t NsA = fA / ds;
    size_t NsB = fB / ds;

    double* wA = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* wB = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* wAds = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* wBds = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* phiA = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* phiB = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* ksi = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* init = (double*)_mm_malloc(size * sizeof(double), alignment);
    double* qA = (double*)_mm_malloc(size * (NsA + 1) * sizeof(double), alignment);
    double* qcA = (double*)_mm_malloc(size * (NsA + 1) * sizeof(double), alignment);
    double* qB = (double*)_mm_malloc(size * (NsB + 1) * sizeof(double), alignment);
    double* qcB = (double*)_mm_malloc(size * (NsB + 1) * sizeof(double), alignment);

    std::memcpy(wA, wA0, size * sizeof(double));
    std::memcpy(wB, wB0, size * sizeof(double));
    c_array<double, 6> cell = {{Lx, Ly, Lz, 0, 0, 0}};
    solver.set_cell_para(cell);
    solver.set_contour_step(ds);

    std::clock_t time = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (size_t itr = 0; itr < (size_t)Nstep; ++itr) {
        calc_ksi(ksi, wA, wB, size, xN);
        array_exp(wAds, wA, 1., -ds / 2, size);
        array_exp(wBds, wB, 1., -ds / 2, size);

        array_set_vals(init, 1, size);
        solve_diffusion_equation(qA, init, wAds, solver, NsA, 1, time);
        solve_diffusion_equation(qcB, init, wBds, solver, NsB, -1, time);
        array_copy(init, qA + NsA * size, size);
        solve_diffusion_equation(qB, init, wBds, solver, NsB, 1, time);
        array_copy(init, qcB, size);
        solve_diffusion_equation(qcA, init, wAds, solver, NsA, -1, time);

        double Q = array_average(qcA, size);
        array_set_vals(phiA, 0, size);
        array_set_vals(phiB, 0, size);
        integrate_phi(phiA, qA, qcA, fA, Q, size, NsA);
        integrate_phi(phiB, qB, qcB, fB, Q, size, NsB);

        double parts[4], maxinc;
        energy_terms(Q, xN, wA, wB, phiA, phiB, ksi, size, parts, &maxinc);
        if (F_out) F_out[itr] = parts[1] + parts[2] + parts[0] + parts[3];
        if (parts_out)
            for (int i = 0; i < 4; ++i) parts_out[4 * itr + i] = parts[i];
        if (maxinc_out) maxinc_out[itr] = maxinc;
        if (Q_out) Q_out[itr] = Q;
        if (itr + 1 == (size_t)Nstep) {
            if (phiA_out) std::memcpy(phiA_out, phiA, size * sizeof(double));
            if (phiB_out) std::memcpy(phiB_out, phiB, size * sizeof(double));
        }
        calc_new_fields(wA, wB, phiA, phiB, ksi, xN, acceptance, size);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (wA_out) std::memcpy(wA_out, wA, size * sizeof(double));
    if (wB_out) std::memcpy(wB_out, wB, size * sizeof(double));
    if (triplet_cpu_seconds) *triplet_cpu_seconds = (double)time / CLOCKS_PER_SEC;

    _mm_free(wA); _mm_free(wB); _mm_free(wAds); _mm_free(wBds);
    _mm_free(phiA); _mm_free(phiB); _mm_free(ksi); _mm_free(init);
    _mm_free(qA); _mm_free(qcA); _mm_free(qB); _mm_free(qcB);
    return std::chrono::duration<double>(t1 - t0).count();
}

// Runs the reference's own template driver diblock_scft_simple_iterate unmodified on the
// physical-size fields wA0/wB0; its stdout is captured into `log` (NUL-terminated,
// truncated to logcap).  The driver also writes `<name>_output.txt`.  Returns the
// reference's std::clock() triplet total.
long ref_run_driver(void* h, long nx, long ny, long nz, double fA, double ds, double xN,
                    double Lx, double Ly, double Lz, double acceptance, long Nstep,
                    const double* wA0, const double* wB0, const char* name, char* log,
                    long logcap) {
    CrysPSSolverBase& solver = *static_cast<RefSolver*>(h)->s;
    size_t size = solver.get_space_size_phy();
    auto init = [size, wA0, wB0](double* wA, double* wB) -> void {
        for (size_t itr = 0; itr < size; ++itr) {
            wA[itr] = wA0[itr];
            wB[itr] = wB0[itr];
        }
    };
    std::ostringstream cap;
    std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
    std::clock_t t = diblock_scft_simple_iterate((size_t)nx, (size_t)ny, (size_t)nz, fA, ds, xN, Lx,
                                                 Ly, Lz, acceptance, (size_t)Nstep,
                                                 std::string(name), solver, init);
    std::cout.rdbuf(old);
    std::string s = cap.str();
    if (log && logcap > 0) {
        size_t n = s.size() < (size_t)(logcap - 1) ? s.size() : (size_t)(logcap - 1);
        std::memcpy(log, s.data(), n);
        log[n] = 0;
    }
    return (long)t;
}

// the reference's text field I/O (src/crysSCFT_sample.cpp:271-292)
void ref_output_fields(const double* phiA, const double* phiB, const double* wA, const double* wB, long size,
                       const char* filename) {
    output_fields(phiA, phiB, wA, wB, (size_t)size, std::string(filename));
}
void ref_input_fields(double* phiA, double* phiB, double* wA, double* wB, long size, const char* filename) {
    input_fields(phiA, phiB, wA, wB, (size_t)size, std::string(filename));
}

void ref_set_num_threads(int n) { omp_set_num_threads(n); }
int ref_get_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
