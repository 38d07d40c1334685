// drivers.h — adaptive estimator drivers (host C++), one per reference entry point.
#pragma once
#include <vector>
#include "engine.h"

namespace mcq {

void run_mc(const mcq_model& m, const mcq_payoff& p, double eps, int n_steps,
            const mcq_mc_cfg& cfg, mcq_result& out);
void run_mc_fixed(const mcq_model& m, const mcq_payoff& p, int n_steps, long long n_paths,
                  uint32_t seed, double& mean, double& var_of_mean);
void run_qmc(const mcq_model& m, const mcq_payoff& p, double eps, int n_steps,
             const mcq_qmc_cfg& cfg, int noise, const Handle* bb, const Handle* pca,
             mcq_result& out);
void run_mlmc(const mcq_model& m, const mcq_payoff& p, double eps, const mcq_mlmc_cfg& cfg,
              mcq_result& out);
void run_mlqmc(const mcq_model& m, const mcq_payoff& p, double eps, const mcq_mlmc_cfg& ml,
               const mcq_qmc_cfg& qc, int noise, const std::vector<const Handle*>& bb_list,
               const std::vector<const Handle*>& pca_list, mcq_result& out);
void cv_pilot(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, int n_steps,
              int N_pilot, uint32_t seed, mcq_cv_pilot_out& out);
void run_mc_cv(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, double beta,
               double eps, int n_steps, const mcq_mc_cfg& cfg, mcq_result& out);
void run_qmc_cv(const mcq_model& main_m, const mcq_payoff& main_p, double E_ctrl, double beta,
                double eps, int n_steps, const mcq_qmc_cfg& cfg, mcq_result& out);
void run_is(const mcq_model& gbm, const mcq_payoff& eur, double z_star, double eps,
            const mcq_mc_cfg& cfg, mcq_result& out);

}  // namespace mcq
