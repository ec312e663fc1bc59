// Host interface of the GRPP engine (engine.cu).
#pragma once

#include <cstdint>
#include <array>
#include <string>
#include <vector>

#include "../../include/libgrpp_b200.h"

namespace grpp {

struct RunOptions {
    int radial_mode = LIBGRPP_B200_RADIAL_PLAIN;
    int raw_so = 0;          // spin-orbit output without the 2/(2L+1) factor (libgrpp_spin_orbit_integrals)
    int fin_nt = 0;          // assembly block size for every task (128, 256, 512); 0: tuning table, else default rule
    int fin_by_class = 0;    // one assembly launch per class, each timed (autotuning)
};

struct RunStats {
    int64_t n_tasks = 0, n_radial = 0, n_mmd = 0, n_entries = 0;
    int64_t fallbacks = 0;
    float ms_total = 0.f, ms_mmd = 0.f, ms_radial = 0.f, ms_final = 0.f, ms_screen = 0.f, ms_predict = 0.f;
    unsigned long long radial_counters[16] = {0};  // RadialCounter slots (radial.cuh)
};

// thread-local last error
void set_error(int code, const std::string &msg);
int last_error();
const char *last_error_message();

// Evaluate all tasks of a batch; outputs are host arrays of libgrpp_b200_batch_output_size doubles.
int run_full_batch(const libgrpp_b200_batch_t *b, const RunOptions &opt, double *arep, double *so_x, double *so_y,
                   double *so_z, RunStats *stats = nullptr);

int64_t batch_output_size(const libgrpp_b200_batch_t *b);

// A batch prepared on the device (inputs uploaded, work lists built, buffers owned):
// execute any number of times, read the outputs, destroy.
struct Plan;
Plan *plan_create(const libgrpp_b200_batch_t *b, const RunOptions &opt);
int plan_run(Plan *P);
void plan_set_counting(Plan *P, bool on);
int plan_outputs(Plan *P, double *arep, double *so_x, double *so_y, double *so_z);
void plan_destroy(Plan *P);
const RunStats *plan_stats(const Plan *P);
int64_t plan_h2d_bytes(const Plan *P);
int set_device(int device);
// per-class block size of the assembly kernel (rows: class key, tasks, ms at 128/256/512, choice)
int autotune_assembly(const libgrpp_b200_batch_t *b, int radial_mode, std::vector<std::array<double, 6>> &rows);
void autotune_reset();
void *host_alloc(size_t bytes);
void host_free(void *p);
int measure_fp64_peak(double *tflops);

// density-contracted gradient (gradient.cuh): one entry per task of the original list
struct GradTaskHost {
    int t_ad, t_au, t_bd, t_bu;  // sub-task indices of (A-1,B) (A+1,B) (A,B-1) (A,B+1); -1 if L = 0
    int la, lb;
    int64_t d_row, d_col;        // basis offsets of shells A and B
};
constexpr int kGradMaxL = 10;      // component table rows L = 0..10 (the engine's kMaxL)
constexpr int kGradTabCart = 66;   // components of L = 10
int run_grad_contract(const libgrpp_b200_batch_t *sub, const RunOptions &opt, const GradTaskHost *tasks,
                      int64_t n_tasks, const int *cart_tab, const double *D, int64_t n_bf, double *out24);

// one-electron integrals (onee.cuh): kind 0 overlap, 1 kinetic (out0), 2 momentum (out0..2)
int run_onee_batch(const libgrpp_b200_batch_t *b, int kind, double *out0, double *out1, double *out2);
// numeric type 1 integrals of a radially local potential per centre: model 0 the centre GRPP's U_L,
// 1..5 nuclear charge models with centre_param[4 * c] = {Z, parameters} (nucmodel.h)
int run_type1_numeric_batch(const libgrpp_b200_batch_t *b, int model, const double *centre_param, double tol,
                            double pair_skip, double *out);

// learned grid-level model (level_model.cuh)
int set_level_model(const float *params);
int level_samples(const libgrpp_b200_batch_t *b, float *features, int8_t *levels, int64_t *n_items);
int mlp_grad(const float *params, const float *X, const int8_t *y, int n, float *grad, float *loss);
int mlp_train(const float *X, const int8_t *y, int64_t n, int epochs, int batch, float lr, uint32_t seed,
              float *params, float *epoch_loss);
int mlp_predict(const float *params, const float *X, int64_t n, int8_t *pred);

}  // namespace grpp
