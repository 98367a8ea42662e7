/*
 * FFTW-API shim header — TEST INFRASTRUCTURE ONLY (oracle).
 *
 * The reference solvers (src/solver_p1.h, src/solver_3m.h, src/solver_Pmmm.h)
 * call six FFTW 3.3.3 entry points.  FFTW is not installed on this machine,
 * so this header declares exactly those entry points (same names, same
 * signatures, same argument meaning) and fftw_shim.c implements them from
 * FFTW's published definitions of the transforms ("What FFTW Really
 * Computes", FFTW 3.3 manual section 4.8):
 *
 *   r2c  : Y[k] = sum_j X[j] exp(-2 pi i j k / n)        (multi-dim, unnormalised)
 *   c2r  : Y[j] = sum_k X[k] exp(+2 pi i j k / n)        (Hermitian input, unnormalised)
 *   REDFT10 (DCT-II) : Y[k] = 2 sum_{j<n} X[j] cos(pi (j+1/2) k / n)
 *   REDFT01 (DCT-III): Y[k] = X[0] + 2 sum_{1<=j<n} X[j] cos(pi j (k+1/2) / n)
 *
 * Call sites this shim serves:
 *   src/solver_p1.h:180-181   fftw_plan_many_dft_r2c / fftw_plan_many_dft_c2r
 *   src/solver_3m.h:277-278   fftw_plan_guru_dft_r2c / fftw_plan_guru_dft_c2r
 *   src/solver_Pmmm.h:190-191 fftw_plan_r2r_3d (REDFT10 / REDFT01)
 *   fftw_execute at src/solver_p1.h:186,201, src/solver_3m.h:290,323,
 *   src/solver_Pmmm.h:195,214
 *
 * Planner flags are accepted and ignored; planning never touches the arrays.
 */
#ifndef CRYSSCFT_ORACLE_FFTW3_SHIM_H
#define CRYSSCFT_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

typedef struct fftw_iodim_do_not_use_me {
    int n;   /* dimension size */
    int is;  /* input stride (in elements of the input type) */
    int os;  /* output stride (in elements of the output type) */
} fftw_iodim;

typedef enum fftw_r2r_kind_do_not_use_me {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_EXHAUSTIVE (1U << 3)

fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                 double* in, const int* inembed, int istride, int idist,
                                 fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                 fftw_complex* in, const int* inembed, int istride, int idist,
                                 double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_guru_dft_r2c(int rank, const fftw_iodim* dims,
                                 int howmany_rank, const fftw_iodim* howmany_dims,
                                 double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_guru_dft_c2r(int rank, const fftw_iodim* dims,
                                 int howmany_rank, const fftw_iodim* howmany_dims,
                                 fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double* in, double* out,
                           fftw_r2r_kind kind0, fftw_r2r_kind kind1, fftw_r2r_kind kind2,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* shim-only helpers used by the oracle tests (not FFTW API) */
void crysscft_shim_dft_1d_direct(int n, const double* in_re, const double* in_im,
                                 double* out_re, double* out_im, int sign);
int crysscft_shim_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
