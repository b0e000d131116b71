// engine.cuh -- simulation context entry points (C++ side of the C-ABI).
#pragma once
#include "../../include/umagnus_b200.h"

namespace umag {
int sim_new(const umag_sim_params* p, const umag_solver_params* sp, umag_sim** out);
int sim_free(umag_sim* s);
int sim_set_m(umag_sim* s, const float* mx, const float* my, const float* mz, int normalise);
int sim_get_m(umag_sim* s, float* mx, float* my, float* mz);
int sim_m_ptrs(umag_sim* s, float** m3);
int sim_torque(umag_sim* s, float* tx, float* ty, float* tz, float* bx, float* by, float* bz);
int sim_steps(umag_sim* s, int n);
int sim_run(umag_sim* s, double seconds, int chunk, long long max_steps);
int sim_get_state(umag_sim* s, umag_solver_state* st);
int sim_plant_status(umag_sim* s, int code);
int sim_set_time(umag_sim* s, double t, double dt);
int sim_average_m(umag_sim* s, double avg[3]);
int sim_use_graph(umag_sim* s, int enable, int steps);
int sim_launches_per_step(umag_sim* s, int* n);
int sim_torque_evals(umag_sim* s, int n);
int sim_energies(umag_sim* s, double E[5]);
int sim_energy_density(umag_sim* s, float* dst);
int sim_relax(umag_sim* s, double threshold);
int sim_set_solver(umag_sim* s, const umag_solver_params* sp);
int sim_set_param(umag_sim* s, int which, const float* values, float mul);
int sim_get_tuning(umag_sim* s, umag_tuning* t);
int sim_set_tuning(umag_sim* s, const umag_tuning* t);
int ens_new(int n, const umag_ens_instance* in, const umag_solver_params* sp, int demag, umag_ens** out);
int ens_new_general(int n, const umag_ens_instance* in, const umag_sim_params* const* general,
                    const umag_solver_params* sp, int demag, umag_ens** out);
int ens_free(umag_ens* e);
int ens_set_m(umag_ens* e, int i, const float* host_m);
int ens_get_m(umag_ens* e, int i, float* host_m);
int ens_get_state(umag_ens* e, int i, umag_solver_state* st);
int ens_run(umag_ens* e, double seconds, int chunk, long long max_replays);
int ens_count(umag_ens* e, int* n_instances, int* n_classes);
int ens_class_info(umag_ens* e, int cls, int N[3], int* n_instances);
int ens_class_general(umag_ens* e, int cls, int* general);
int ens_get_tuning(umag_ens* e, int cls, umag_tuning* t);
int ens_set_tuning(umag_ens* e, int cls, const umag_tuning* t);
int adj_new(const umag_adj_params* p, umag_adj** out);
int adj_free(umag_adj* a);
int adj_forward(umag_adj* a, const float* m0, const float* Ms, float A, float K1, const float Bext[3], double* loss);
int adj_final_m(umag_adj* a, float* m);
int adj_backward(umag_adj* a, float* gMs, float* gm0, double* gA, double* gK1, double gB[3]);
int adj_forward_regions(umag_adj* a, const float* m0, const float* Ms, const float* A, const float* K1,
                        const float* Bext, double* loss);
int adj_backward_regions(umag_adj* a, float* gMs, float* gm0, double* gA, double* gK1, double* gB);
}  // namespace umag
