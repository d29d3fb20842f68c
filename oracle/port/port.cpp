// TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// Host restatement of the reference's MPPI and PR-MPPI kernels (src/kernels.cu,
// src/prmppi_kernels.cu) and of the host tails of the controllers
// (src/mppi_controller.cu, src/prmppi_controller.cu), on top of the model in
// model.hpp. Each function is exported with C linkage for ctypes and evaluates
// in FP32 (prec == 32, reference arithmetic) or FP64 (prec == 64, transcription).
// Random perturbations are inputs (materialised from the Philox streams by the
// orc_*_noise functions); the in-rollout environment noise is drawn from the same
// Philox streams as the product.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <boost/math/distributions/beta.hpp> // oracle/stubs (boost is absent here)

#include "gate_model.hpp"
#include "model.hpp"

using namespace orc;

namespace
{

template <typename R> MppiCosts<R> mppiCosts(const dr_mppi_config& c)
{
    return MppiCosts<R>{c.coll_dist_factor, c.boundary_cost, c.boundary_threshold_factor, c.outside_cost,
                        c.win_cost,         c.opp_win_cost, c.final_adv_weight,          c.final_opp_adv_weight};
}

template <typename R> PrCosts<R> prCosts(const dr_prmppi_config& c)
{
    return PrCosts<R>{c.coll_dist_factor, c.boundary_cost,    c.boundary_threshold_factor, c.win_cost,
                      c.opp_win_cost,     c.final_adv_weight, c.final_opp_adv_weight,      c.safety_weight};
}

inline int mk(const dr_mppi_config& c)
{
    return c.use_splines ? c.n_knots : c.n_timesteps;
}

// fullRolloutKernel, src/kernels.cu:34-171 (one loop iteration per thread s), for either
// model: EnvT / StateT are Env / State of model.hpp or of gate_model.hpp, whose
// environmentStep, stateCost and finalCost are found by argument-dependent lookup.
template <typename R, typename EnvT, typename StateT, typename FlagsT, typename S0>
void mppiRolloutT(const EnvT& env, const FlagsT& flags, const dr_mppi_config& mc, const S0& s0, const float* belief0, const float* nominal,
                  const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed, int* branchTime)
{
    const int K = mc.n_samples, T = mc.n_timesteps, M = mk(mc), nth = env.nth;
    const R minConf = mc.min_confidence;
    MppiCosts<R> cc = mppiCosts<R>(mc);
    R initBelief[DR_MAX_THETA];
    for (int th = 0; th < nth; th++)
        initBelief[th] = belief0[th];

#pragma omp parallel for schedule(dynamic, 16)
    for (int s = 0; s < K; s++)
    {
        Branch<R> first;
        initBranchState(first, initBelief, nth, minConf);
        for (int th = 0; th < nth; th++)
        {
            costsTrue[th * K + s] = INFINITY;
            branchUsed[th * K + s] = first.predTheta;
            branchTime[th * K + s] = first.branchingTime;
        }
        for (int th = 0; th < nth; th++)
        {
            if (!branchCompatibleWithModel(first.predTheta, th))
                continue;
            StateT st = StateT::from(s0);
            Branch<R> bs = first;
            R cost = R(0);
            bool stop = false;
            R decay = R(1);
            int tOrigin = 0;
            EnvNoise rng(seed, (uint32_t)s, (uint32_t)th << 16, step, S_MPPI_ROLL_ENV);
            for (int t = 0; t < T && !stop; t++)
            {
                rng.begin_step((uint32_t)t);
                int local = t - tOrigin;
                int b = bs.predTheta;
                R ego[DIM];
                if (mc.use_splines)
                {
                    const float* Brow = B + local * M;
                    for (int d = 0; d < DIM; d++)
                    {
                        R sum = R(0);
                        for (int m = 0; m < M; m++)
                        {
                            R nom = nominal[(b * M + m) * DIM + d];
                            R nz = noise[((size_t)(b * M + m) * K + s) * DIM + d];
                            sum += (R)Brow[m] * (nom + nz);
                        }
                        ego[d] = sum;
                    }
                }
                else
                    for (int d = 0; d < DIM; d++)
                    {
                        R nom = nominal[(b * T + local) * DIM + d];
                        R nz = noise[((size_t)(b * T + local) * K + s) * DIM + d];
                        ego[d] = nom + nz;
                    }
                bool branched = false;
                int term = environmentStep(t, th, env, ego, flags, st, bs, branched, minConf, rng);
                if (branched)
                    tOrigin = t + 1;
                stop = (term != TERM_NONE);
                cost += stateCost(st, env, cc) * decay;
                decay *= (R)DECAY;
            }
            cost += finalCost(st, env, cc.finalAdvWeight, cc.finalOppAdvWeight);
            costsTrue[th * K + s] = (double)cost;
            branchTime[th * K + s] = bs.branchingTime;
            branchUsed[th * K + s] = bs.predTheta;
        }
    }
}

template <typename R>
void mppiRollout(const dr_env_config& ec, const dr_mppi_config& mc, const dr_sim_state& s0, const float* belief0, const float* nominal,
                 const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed, int* branchTime)
{
    Env<R> env(ec);
    const StepFlags flags{true, true, true, true, true};
    mppiRolloutT<R, Env<R>, State<R>>(env, flags, mc, s0, belief0, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
}

// the gate race: environmentStep<true, true, false> (kernels.cu:141-143; addMargin off)
template <typename R>
void gateRollout(const dr_gate_env_config& ec, const dr_mppi_config& mc, const dr_gate_state& s0, const float* belief0, const float* nominal,
                 const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed, int* branchTime)
{
    gate::Env<R> env(ec);
    const gate::Flags flags{true, true, false, true, true, mc.gate_traversal_margin};
    mppiRolloutT<R, gate::Env<R>, gate::State<R>>(env, flags, mc, s0, belief0, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
}

// coefficient of sample s for (branch plan b, knot/timestep k): kernels.cu:252-279
template <typename R>
R sampleCoeff(const dr_mppi_config& mc, int nth, const R* belief, int b, int k, int s, int K, const int* branchUsed, const int* branchTime)
{
    R coeff = R(0);
    for (int th = 0; th < nth; th++)
    {
        if (belief[th] <= R(0))
            continue;
        if (!branchCompatibleWithModel(b, th))
            continue;
        int pt = branchUsed[th * K + s];
        int bt = branchTime[th * K + s];
        bool c = mc.use_splines ? splineSampleContributed(b, k, bt, pt, mc.n_timesteps, mc.n_knots, mc.knots)
                                : sampleContributed(b, k, bt, pt, mc.n_timesteps);
        if (c)
            coeff += belief[th];
    }
    return coeff;
}

// aggregateBranchCostsKernel (kernels.cu:175-217), computeMaskedMinCostsKernel
// (221-301), weightedAverageKernelUnified (307-408), interpolateSplineKernel
// (411-431) and clampNominalKernel (434-456), in launch order
// (mppi_controller.cu:299-345). blockorder != 0 sums the weighted average the way a
// 256-thread block does (strided partials, then a halving tree).
template <typename R>
void mppiUpdate(int nth, float maxAccelEgo, const dr_mppi_config& mc, const float* belief0, const double* costsTrueIn, const int* branchUsed,
                const int* branchTime, const float* noise, const float* B, double* knotsIO, double* denseOut, double* minCostsOut, double* nuOut,
                double* costsOut, int blockorder)
{
    const int K = mc.n_samples, T = mc.n_timesteps, M = mk(mc), nbp = nth + 1;
    R belief[DR_MAX_THETA];
    for (int th = 0; th < nth; th++)
        belief[th] = belief0[th];
    std::vector<R> costsTrue((size_t)nth * K), costs((size_t)nbp * K);
    for (size_t i = 0; i < costsTrue.size(); i++)
        costsTrue[i] = (R)costsTrueIn[i];
    // aggregate
    for (int b = 0; b < nbp; b++)
        for (int s = 0; s < K; s++)
        {
            R num = R(0), den = R(0);
            for (int th = 0; th < nth; th++)
            {
                if (!branchCompatibleWithModel(b, th))
                    continue;
                R c = costsTrue[th * K + s];
                if (!isfinite(c))
                    continue;
                R w = belief[th];
                num += w * c;
                den += w;
            }
            costs[b * K + s] = (den > R(1e-30f)) ? (num / den) : (R)INFINITY;
        }
    if (costsOut)
        for (size_t i = 0; i < costs.size(); i++)
            costsOut[i] = (double)costs[i];
    // masked min
    const int initPred = findConfident(belief, nth, (R)mc.min_confidence);
    std::vector<R> minCosts((size_t)nbp * M);
#pragma omp parallel for collapse(2)
    for (int b = 0; b < nbp; b++)
        for (int k = 0; k < M; k++)
        {
            R mn = INFINITY;
            if (branchCompatibleWithInitialModel(b, initPred))
                for (int s = 0; s < K; s++)
                {
                    R coeff = sampleCoeff(mc, nth, belief, b, k, s, K, branchUsed, branchTime);
                    if (coeff > (R)MIN_COEFF_THRESHOLD)
                    {
                        R c = costs[b * K + s];
                        if (c < mn)
                            mn = c;
                    }
                }
            minCosts[b * M + k] = mn;
        }
    // weighted average
    std::vector<R> knots((size_t)nbp * M * DIM);
    for (size_t i = 0; i < knots.size(); i++)
        knots[i] = (R)knotsIO[i];
    std::vector<R> nu(nbp, R(0));
    const R lambda = mc.inv_temperature;
#pragma omp parallel for collapse(3)
    for (int b = 0; b < nbp; b++)
        for (int k = 0; k < M; k++)
            for (int d = 0; d < DIM; d++)
            {
                const int NT = 256;
                R pnum[NT], pden[NT];
                for (int i = 0; i < NT; i++)
                    pnum[i] = pden[i] = R(0);
                R minC = minCosts[b * M + k];
                if (!isinf(minC))
                    for (int s = 0; s < K; s++)
                    {
                        R coeff = sampleCoeff(mc, nth, belief, b, k, s, K, branchUsed, branchTime);
                        if (coeff > (R)MIN_COEFF_THRESHOLD)
                        {
                            R cost = costs[b * K + s];
                            R w = exp(-(cost - minC) / lambda);
                            R eps = noise[((size_t)(b * M + k) * K + s) * DIM + d];
                            int slot = blockorder ? (s % NT) : 0;
                            pnum[slot] += w * coeff * eps;
                            pden[slot] += w * coeff;
                        }
                    }
                if (blockorder)
                    for (int stride = NT / 2; stride > 0; stride >>= 1)
                        for (int i = 0; i < stride; i++)
                        {
                            pnum[i] += pnum[i + stride];
                            pden[i] += pden[i + stride];
                        }
                if (pden[0] > R(1e-30f))
                    knots[(b * M + k) * DIM + d] += pnum[0] / pden[0];
                if (k == 0 && d == 0)
                    nu[b] = pden[0];
            }
    for (int i = 0; i < nbp * M; i++)
        minCostsOut[i] = (double)minCosts[i];
    for (int b = 0; b < nbp; b++)
        nuOut[b] = (double)nu[b];
    // interpolate (spline mode): dense = B * knots, before the clamp
    std::vector<R> dense((size_t)nbp * T * DIM);
    if (mc.use_splines)
        for (int b = 0; b < nbp; b++)
            for (int t = 0; t < T; t++)
                for (int d = 0; d < DIM; d++)
                {
                    R sum = R(0);
                    for (int m = 0; m < M; m++)
                        sum += (R)B[t * M + m] * knots[(b * M + m) * DIM + d];
                    dense[(b * T + t) * DIM + d] = sum;
                }
    // clamp (knots in spline mode, the dense nominal otherwise)
    const R maxAccel = maxAccelEgo; // Env::getMaxAccel (mppi_controller.cu:345)
    for (int v = 0; v < nbp * M; v++)
    {
        R sq = R(0);
        for (int d = 0; d < DIM; d++)
            sq += knots[v * DIM + d] * knots[v * DIM + d];
        R maxSq = maxAccel * maxAccel;
        if (sq > maxSq)
        {
            R scale = maxAccel / sqrt(sq);
            for (int d = 0; d < DIM; d++)
                knots[v * DIM + d] *= scale;
        }
    }
    if (!mc.use_splines)
        dense = knots;
    for (size_t i = 0; i < knots.size(); i++)
        knotsIO[i] = (double)knots[i];
    for (size_t i = 0; i < dense.size(); i++)
        denseOut[i] = (double)dense[i];
}

// sampleModelFromBelief, state.h:118-131 (uniform from the Philox stream).
template <typename R> int sampleModel(const R* belief, int nth, float u)
{
    R cdf = R(0);
    for (int k = 0; k < nth; k++)
    {
        cdf += belief[k];
        if ((R)u <= cdf)
            return k;
    }
    return nth - 1;
}

// verifyNominalFailureKernel, src/kernels.cu:488-551, for either model (as mppiRolloutT).
template <typename R, typename EnvT, typename StateT, typename FlagsT, typename S0>
void mppiVerifyT(const EnvT& env, const FlagsT& flags, const dr_mppi_config& mc, const S0& s0, const float* belief0, const double* plan, uint64_t seed,
                 uint64_t step, int planId, unsigned* failCount, int* failTime, int* thetasOut)
{
    const int V = mc.n_verif_samples, T = mc.n_timesteps, H = mc.verif_horizon, nth = env.nth;
    const R minConf = mc.min_confidence;
    R initBelief[DR_MAX_THETA];
    for (int th = 0; th < nth; th++)
        initBelief[th] = belief0[th];
    std::vector<R> nominal((size_t)(nth + 1) * T * DIM);
    for (size_t i = 0; i < nominal.size(); i++)
        nominal[i] = (R)plan[i];
    const Key key(seed);
    std::vector<int> ft(V, -1);
#pragma omp parallel for schedule(dynamic, 64)
    for (int v = 0; v < V; v++)
    {
        StateT st = StateT::from(s0);
        Branch<R> bs;
        initBranchState(bs, initBelief, nth, minConf);
        float u = uniform_from_word(draw(key, (uint32_t)v, (uint32_t)planId, step, S_VERIF_THETA, 0).v[0]);
        int theta = sampleModel(bs.belief, nth, u);
        if (thetasOut)
            thetasOut[v] = theta;
        EnvNoise rng(seed, (uint32_t)v, (uint32_t)planId << 16, step, S_VERIF_ENV);
        int tOrigin = 0, t = 0;
        bool failed = false;
        for (; t < H; t++)
        {
            rng.begin_step((uint32_t)t);
            int local = t - tOrigin;
            int b = bs.predTheta;
            R ego[DIM];
            for (int d = 0; d < DIM; d++)
                ego[d] = nominal[(b * T + local) * DIM + d];
            bool branched = false;
            int term = environmentStep(t, theta, env, ego, flags, st, bs, branched, minConf, rng);
            if (branched)
                tOrigin = t + 1;
            if (term == TERM_LOSE)
            {
                failed = true;
                break;
            }
            else if (term == TERM_WIN || term == TERM_OPP_WIN)
                break;
        }
        if (failed)
            ft[v] = t;
    }
    for (int t = 0; t < T; t++)
        failCount[t] = 0;
    for (int v = 0; v < V; v++)
    {
        if (ft[v] >= 0)
            failCount[ft[v]]++;
        if (failTime)
            failTime[v] = ft[v];
    }
}

template <typename R>
void mppiVerify(const dr_env_config& ec, const dr_mppi_config& mc, const dr_sim_state& s0, const float* belief0, const double* plan, uint64_t seed,
                uint64_t step, int planId, unsigned* failCount, int* failTime, int* thetasOut)
{
    Env<R> env(ec);
    const StepFlags flags{true, true, false, true, true};
    mppiVerifyT<R, Env<R>, State<R>>(env, flags, mc, s0, belief0, plan, seed, step, planId, failCount, failTime, thetasOut);
}

// the gate race: environmentStep<true, true, false, false> (kernels.cu:529-531)
template <typename R>
void gateVerify(const dr_gate_env_config& ec, const dr_mppi_config& mc, const dr_gate_state& s0, const float* belief0, const double* plan,
                uint64_t seed, uint64_t step, int planId, unsigned* failCount, int* failTime, int* thetasOut)
{
    gate::Env<R> env(ec);
    const gate::Flags flags{true, true, false, false, true, mc.gate_traversal_margin};
    mppiVerifyT<R, gate::Env<R>, gate::State<R>>(env, flags, mc, s0, belief0, plan, seed, step, planId, failCount, failTime, thetasOut);
}

// PRMPPIfullRolloutKernel, src/prmppi_kernels.cu:55-130 (one iteration per (nom/rob, p, s)).
template <typename R>
void prRollout(const dr_env_config& ec, const dr_prmppi_config& pc, const dr_sim_state& s0, const double* nom, const double* rob, const float* noise,
               const int* thetas, uint64_t seed, uint64_t step, double* costNom, double* costRob)
{
    Env<R> env(ec);
    const int K = pc.n_samples, T = pc.n_timesteps, P = pc.P;
    PrCosts<R> cc = prCosts<R>(pc);
    std::vector<R> nomR((size_t)T * DIM), robR((size_t)T * DIM);
    for (int i = 0; i < T * DIM; i++)
    {
        nomR[i] = (R)nom[i];
        robR[i] = (R)rob[i];
    }
    const StepFlags flags{false, false, true, true, false};
    const long total = (long)K * P;
#pragma omp parallel for schedule(dynamic, 16)
    for (long tid = 0; tid < 2 * total; tid++)
    {
        bool robust = tid >= total;
        long idx = robust ? tid - total : tid;
        int p = (int)(idx / K), s = (int)(idx % K);
        const std::vector<R>& nominal = robust ? robR : nomR;
        int theta = thetas[p];
        State<R> st = State<R>::from(s0);
        Branch<R> bs{};
        R running = R(0), safe = -INFINITY, decay = R(1);
        bool stop = false;
        EnvNoise rng(seed, (uint32_t)s, ((((uint32_t)robust << 8) | (uint32_t)p) << 16), step, S_PR_ROLL_ENV);
        for (int t = 0; t < T && !stop; t++)
        {
            rng.begin_step((uint32_t)t);
            R ego[DIM];
            for (int d = 0; d < DIM; d++)
                ego[d] = nominal[t * DIM + d] + (R)noise[((size_t)t * K + s) * DIM + d];
            bool branched = false;
            int term = environmentStep(t, theta, env, ego, flags, st, bs, branched, R(0), rng);
            stop = (term != TERM_NONE);
            running += decay * prStateCost(st, env, cc);
            safe = fmax(safe, prSafetyCost(st, env, cc));
            decay *= (R)DECAY;
        }
        running += finalCost(st, env, cc.finalAdvWeight, cc.finalOppAdvWeight);
        double* out = robust ? costRob : costNom;
        out[(idx)*2 + 0] = (double)running;
        out[(idx)*2 + 1] = (double)safe;
    }
}

// PRMPPIcostAvgKernel (prmppi_kernels.cu:134-166), PRMPPIcomputeMinCostsKernel
// (169-199) and PRMPPIWeightedAverageKernel (204-282). costNom/costRob are updated
// in place at p = 0 like the reference.
template <typename R>
void prUpdate(const dr_prmppi_config& pc, double* costNomIO, double* costRobIO, const float* noise, const double* nom, const double* rob,
              const float* invTemps, double* minCostsOut, double* cand1, double* cand2, double* newRob, double* nuOut, int blockorder)
{
    const int K = pc.n_samples, T = pc.n_timesteps, P = pc.P;
    std::vector<R> cn((size_t)P * K * 2), cr((size_t)P * K * 2);
    for (size_t i = 0; i < cn.size(); i++)
    {
        cn[i] = (R)costNomIO[i];
        cr[i] = (R)costRobIO[i];
    }
    const R sw = pc.safety_weight;
    for (int which = 0; which < 2; which++)
    {
        std::vector<R>& c = which == 0 ? cn : cr;
        for (int s = 0; s < K; s++)
        {
            R avg = R(0), maxSafe = -INFINITY;
            for (int p = 0; p < P; p++)
            {
                size_t off = ((size_t)p * K + s) * 2;
                avg += c[off];
                maxSafe = fmax(maxSafe, c[off + 1]);
            }
            avg /= (R)P;
            c[s * 2] = avg + ((maxSafe > R(0)) ? sw : R(0));
            c[s * 2 + 1] = maxSafe;
        }
    }
    for (size_t i = 0; i < cn.size(); i++)
    {
        costNomIO[i] = (double)cn[i];
        costRobIO[i] = (double)cr[i];
    }
    R minCosts[3];
    for (int which = 0; which < 3; which++)
    {
        const R* arr = which == 0 ? cn.data() : (which == 1 ? cr.data() : cr.data() + 1);
        R v = INFINITY;
        for (int i = 0; i < K; i++)
            v = fmin(v, arr[i * 2]);
        minCosts[which] = v;
        minCostsOut[which] = (double)v;
    }
    for (int which = 0; which < 3; which++)
    {
        const double* nominal = which == 0 ? nom : rob;
        const R* arr = which == 0 ? cn.data() : (which == 1 ? cr.data() : cr.data() + 1);
        double* out = which == 0 ? cand1 : (which == 1 ? cand2 : newRob);
        R lambda = invTemps[which];
        for (int t = 0; t < T; t++)
            for (int d = 0; d < DIM; d++)
            {
                const int NT = 256;
                R pnum[NT], pden[NT];
                for (int i = 0; i < NT; i++)
                    pnum[i] = pden[i] = R(0);
                R nomv = (R)nominal[t * DIM + d];
                for (int i = 0; i < K; i++)
                {
                    R cost = arr[2 * i];
                    R w = exp(-(cost - minCosts[which]) / lambda);
                    R u = nomv + (R)noise[((size_t)t * K + i) * DIM + d];
                    int slot = blockorder ? (i % NT) : 0;
                    pnum[slot] += w * u;
                    pden[slot] += w;
                }
                if (blockorder)
                    for (int stride = NT / 2; stride > 0; stride >>= 1)
                        for (int i = 0; i < stride; i++)
                        {
                            pnum[i] += pnum[i + stride];
                            pden[i] += pden[i + stride];
                        }
                R value = (pden[0] > R(1e-30f)) ? pnum[0] / pden[0] : nomv;
                out[t * DIM + d] = (double)value;
                if (t == 0 && d == 0)
                    nuOut[which] = (double)pden[0];
            }
    }
}

// PRMPPIcomputeCandidateCostKernel (prmppi_kernels.cu:285-347) when stream ==
// S_PR_CAND_ENV, or the rollout of PRMPPIcomputeSafeCostKernel (350-393) when
// stream == S_PR_SAFE_ENV: full cost and max safety cost of each (cand, p).
template <typename R>
void prCandidates(const dr_env_config& ec, const dr_prmppi_config& pc, const dr_sim_state& s0, const double* cand1, const double* cand2, const int* thetas,
                  uint64_t seed, uint64_t step, uint32_t stream, double* fullCost, double* safeCost)
{
    Env<R> env(ec);
    const int T = pc.n_timesteps, P = pc.P;
    PrCosts<R> cc = prCosts<R>(pc);
    const StepFlags flags{false, false, true, true, false};
    for (int tid = 0; tid < 2 * P; tid++)
    {
        bool second = tid >= P;
        int p = second ? tid - P : tid;
        const double* nominal = second ? cand2 : cand1;
        State<R> st = State<R>::from(s0);
        Branch<R> bs{};
        R cost = R(0), safe = -INFINITY, decay = R(1);
        bool stop = false;
        EnvNoise rng(seed, (uint32_t)p, (uint32_t)second << 16, step, stream);
        for (int t = 0; t < T && !stop; ++t)
        {
            rng.begin_step((uint32_t)t);
            R ego[DIM];
            for (int d = 0; d < DIM; ++d)
                ego[d] = (R)nominal[t * DIM + d];
            bool branched = false;
            int term = environmentStep(t, thetas[p], env, ego, flags, st, bs, branched, R(0), rng);
            stop = (term != TERM_NONE);
            cost += decay * prStateCost(st, env, cc);
            decay *= (R)DECAY;
            safe = fmax(safe, prSafetyCost(st, env, cc));
        }
        cost += finalCost(st, env, cc.finalAdvWeight, cc.finalOppAdvWeight);
        if (safe > R(0))
            cost += cc.safetyWeight;
        fullCost[tid] = (double)cost;
        safeCost[tid] = (double)safe;
    }
}

} // namespace

extern "C" {

// ---- random streams ------------------------------------------------------------------

// Control perturbation of an MPPI step in the reference layout noise[nbp][M][K][DIM]
// (kernels.cu:28).
void orc_mppi_noise(uint64_t seed, uint64_t step, int nbp, int M, int K, const float* sigma, float* out)
{
    const Key key(seed);
    for (int b = 0; b < nbp; b++)
        for (int k = 0; k < M; k++)
            for (int s = 0; s < K; s++)
            {
                Philox4 r = draw(key, (uint32_t)s, (uint32_t)(b * M + k), step, S_MPPI_EPS, 0);
                for (int d = 0; d < DIM; d++)
                    out[((size_t)(b * M + k) * K + s) * DIM + d] = sigma[d] * normal_from_uniform(uniform_from_word(r.v[d]));
            }
}

// PR-MPPI perturbation noise[T][K][DIM] (prmppi_kernels.cu:17).
void orc_pr_noise(uint64_t seed, uint64_t step, int T, int K, const float* sigma, float* out)
{
    const Key key(seed);
    for (int t = 0; t < T; t++)
        for (int s = 0; s < K; s++)
        {
            Philox4 r = draw(key, (uint32_t)s, (uint32_t)t, step, S_PR_EPS, 0);
            for (int d = 0; d < DIM; d++)
                out[((size_t)t * K + s) * DIM + d] = sigma[d] * normal_from_uniform(uniform_from_word(r.v[d]));
        }
}

// PRMPPIsampleThetaValues, prmppi_kernels.cu:23-51.
void orc_pr_thetas(uint64_t seed, uint64_t step, int P, int nth, const float* belief, int* thetas)
{
    const Key key(seed);
    for (int p = 0; p < P; p++)
    {
        float u = uniform_from_word(draw(key, (uint32_t)p, 0u, step, S_PR_THETA, 0).v[0]);
        float accum = 0.0f;
        int theta = nth - 1;
        for (int i = 0; i < nth; i++)
        {
            accum += belief[i];
            if (u <= accum)
            {
                theta = i;
                break;
            }
        }
        thetas[p] = theta;
    }
}

void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t* out)
{
    Philox4 r = philox4x32_10(c0, c1, c2, c3, k0, k1);
    for (int i = 0; i < 4; i++)
        out[i] = r.v[i];
}

void orc_normals_from_words(const uint32_t* w, int n, float* out)
{
    for (int i = 0; i < n; i++)
        out[i] = normal_from_uniform(uniform_from_word(w[i]));
}

float orc_series_logf(float x)
{
    return series_logf(x);
}

// ---- MPPI pieces ----------------------------------------------------------------------

int orc_mppi_rollout(int prec, const dr_env_config* ec, const dr_mppi_config* mc, const dr_sim_state* s0, const float* belief, const float* nominal,
                     const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed, int* branchTime)
{
    if (prec == 64)
        mppiRollout<double>(*ec, *mc, *s0, belief, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
    else
        mppiRollout<float>(*ec, *mc, *s0, belief, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
    return 0;
}

int orc_mppi_update(int prec, const dr_env_config* ec, const dr_mppi_config* mc, const float* belief, const double* costsTrue, const int* branchUsed,
                    const int* branchTime, const float* noise, const float* B, double* knotsIO, double* denseOut, double* minCosts, double* nu,
                    double* costsOut, int blockorder)
{
    if (prec == 64)
        mppiUpdate<double>(ec->n_theta, ec->max_accel[0], *mc, belief, costsTrue, branchUsed, branchTime, noise, B, knotsIO, denseOut, minCosts, nu,
                           costsOut, blockorder);
    else
        mppiUpdate<float>(ec->n_theta, ec->max_accel[0], *mc, belief, costsTrue, branchUsed, branchTime, noise, B, knotsIO, denseOut, minCosts, nu,
                          costsOut, blockorder);
    return 0;
}

// ---- gate race ------------------------------------------------------------------------

int orc_gate_rollout(int prec, const dr_gate_env_config* ec, const dr_mppi_config* mc, const dr_gate_state* s0, const float* belief,
                     const float* nominal, const float* noise, const float* B, uint64_t seed, uint64_t step, double* costsTrue, int* branchUsed,
                     int* branchTime)
{
    if (prec == 64)
        gateRollout<double>(*ec, *mc, *s0, belief, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
    else
        gateRollout<float>(*ec, *mc, *s0, belief, nominal, noise, B, seed, step, costsTrue, branchUsed, branchTime);
    return 0;
}

int orc_gate_update(int prec, const dr_gate_env_config* ec, const dr_mppi_config* mc, const float* belief, const double* costsTrue,
                    const int* branchUsed, const int* branchTime, const float* noise, const float* B, double* knotsIO, double* denseOut,
                    double* minCosts, double* nu, double* costsOut, int blockorder)
{
    const float maxAccel = ec->max_accel[ec->i_mppi];
    if (prec == 64)
        mppiUpdate<double>(ec->n_theta, maxAccel, *mc, belief, costsTrue, branchUsed, branchTime, noise, B, knotsIO, denseOut, minCosts, nu, costsOut,
                           blockorder);
    else
        mppiUpdate<float>(ec->n_theta, maxAccel, *mc, belief, costsTrue, branchUsed, branchTime, noise, B, knotsIO, denseOut, minCosts, nu, costsOut,
                          blockorder);
    return 0;
}

int orc_gate_verify(int prec, const dr_gate_env_config* ec, const dr_mppi_config* mc, const dr_gate_state* s0, const float* belief, const double* plan,
                    uint64_t seed, uint64_t step, int planId, unsigned* failCount, int* failTime, int* thetas)
{
    if (prec == 64)
        gateVerify<double>(*ec, *mc, *s0, belief, plan, seed, step, planId, failCount, failTime, thetas);
    else
        gateVerify<float>(*ec, *mc, *s0, belief, plan, seed, step, planId, failCount, failTime, thetas);
    return 0;
}

// environmentStep on the gate race (the reference's flags as arguments), for unit tests
int orc_gate_env_step(int prec, const dr_gate_env_config* ec, int trueTheta, const float* action, dr_gate_state* state, float* belief,
                      int updateBelief, int considerBranching, float minConfidence, int addMargin, float gateMargin, int loseOnOppWin, int applyNoise,
                      uint64_t seed, uint64_t step, int t)
{
    auto run = [&](auto zero) -> int
    {
        using R = decltype(zero);
        gate::Env<R> env(*ec);
        gate::State<R> st = gate::State<R>::from(*state);
        Branch<R> bs;
        R b0[DR_MAX_THETA];
        for (int th = 0; th < ec->n_theta; th++)
            b0[th] = belief[th];
        initBranchState(bs, b0, ec->n_theta, (R)minConfidence);
        gate::Flags f{updateBelief != 0, considerBranching != 0, addMargin != 0, loseOnOppWin != 0, applyNoise != 0, gateMargin};
        EnvNoise rng(seed, 0u, 0u, step, S_ENV_STEP);
        rng.begin_step(0);
        R ego[DIM] = {(R)action[0], (R)action[1]};
        bool branched = false;
        int term = environmentStep(t, trueTheta, env, ego, f, st, bs, branched, (R)minConfidence, rng);
        st.to(*state);
        for (int th = 0; th < ec->n_theta; th++)
            belief[th] = (float)bs.belief[th];
        return term;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

// stateCost and finalCost of a gate-race state (for unit tests)
void orc_gate_costs(const dr_gate_env_config* ec, const dr_mppi_config* mc, const dr_gate_state* s, float* out2)
{
    gate::Env<float> env(*ec);
    gate::State<float> st = gate::State<float>::from(*s);
    MppiCosts<float> m = mppiCosts<float>(*mc);
    out2[0] = stateCost(st, env, m);
    out2[1] = finalCost(st, env, m.finalAdvWeight, m.finalOppAdvWeight);
}

int orc_mppi_verify(int prec, const dr_env_config* ec, const dr_mppi_config* mc, const dr_sim_state* s0, const float* belief, const double* plan,
                    uint64_t seed, uint64_t step, int planId, unsigned* failCount, int* failTime, int* thetas)
{
    if (prec == 64)
        mppiVerify<double>(*ec, *mc, *s0, belief, plan, seed, step, planId, failCount, failTime, thetas);
    else
        mppiVerify<float>(*ec, *mc, *s0, belief, plan, seed, step, planId, failCount, failTime, thetas);
    return 0;
}

// buildSplineMatrix, src/mppi_controller.cu:56-141 (float arithmetic as in the reference).
void orc_spline_matrix(int T, int M, const int* knots, float* Bout)
{
    std::vector<float> B((size_t)T * M, 0.0f);
    std::vector<int> tau(knots, knots + M);
    std::vector<float> h(M > 1 ? M - 1 : 0);
    for (int j = 0; j < M - 1; j++)
        h[j] = float(tau[j + 1] - tau[j]);
    for (int basis = 0; basis < M; basis++)
    {
        std::vector<float> y(M, 0.0f);
        y[basis] = 1.0f;
        std::vector<float> m(M, 0.0f);
        if (M > 2)
        {
            const int N = M - 2;
            std::vector<float> a(N), b(N), c(N), d(N);
            for (int i = 0; i < N; ++i)
            {
                const int j = i + 1;
                a[i] = h[j - 1];
                b[i] = 2.0f * (h[j - 1] + h[j]);
                c[i] = h[j];
                d[i] = 6.0f * ((y[j + 1] - y[j]) / h[j] - (y[j] - y[j - 1]) / h[j - 1]);
            }
            for (int i = 1; i < N; ++i)
            {
                float w = a[i] / b[i - 1];
                b[i] -= w * c[i - 1];
                d[i] -= w * d[i - 1];
            }
            std::vector<float> x(N);
            x[N - 1] = d[N - 1] / b[N - 1];
            for (int i = N - 2; i >= 0; --i)
                x[i] = (d[i] - c[i] * x[i + 1]) / b[i];
            for (int i = 0; i < N; ++i)
                m[i + 1] = x[i];
        }
        int seg = 0;
        for (int t = 0; t < T; ++t)
        {
            float val = 0.0f;
            if (t <= tau.front())
                val = y.front();
            else if (t >= tau.back())
                val = y.back();
            else
            {
                while (!(tau[seg] <= t && t <= tau[seg + 1]))
                    ++seg;
                const float x0 = float(tau[seg]);
                const float x1 = float(tau[seg + 1]);
                const float hh = x1 - x0;
                const float A = (x1 - t) / hh;
                const float BB = (t - x0) / hh;
                val = m[seg] * (A * A * A - A) * (hh * hh) / 6.0f + m[seg + 1] * (BB * BB * BB - BB) * (hh * hh) / 6.0f + y[seg] * A + y[seg + 1] * BB;
            }
            B[t * M + basis] = val;
        }
    }
    std::memcpy(Bout, B.data(), B.size() * sizeof(float));
}

// shiftSplineKernel, src/kernels.cu:461-486 (in place on branch branchIdx).
void orc_shift_spline(const dr_mppi_config* mc, const float* B, double* knots, int branchIdx, int prec)
{
    const int M = mc->n_knots, T = mc->n_timesteps;
    std::vector<double> src(knots, knots + (size_t)(branchIdx + 1) * M * DIM);
    for (int newm = 0; newm < M; newm++)
        for (int d = 0; d < DIM; d++)
        {
            int tEval = mc->knots[newm] + 1;
            if (tEval >= T)
                tEval = T - 1;
            if (prec == 64)
            {
                double sum = 0.0;
                for (int m = 0; m < M; m++)
                    sum += (double)B[tEval * M + m] * src[(branchIdx * M + m) * DIM + d];
                knots[(branchIdx * M + newm) * DIM + d] = sum;
            }
            else
            {
                float sum = 0.0f;
                for (int m = 0; m < M; m++)
                    sum += B[tEval * M + m] * (float)src[(branchIdx * M + m) * DIM + d];
                knots[(branchIdx * M + newm) * DIM + d] = sum;
            }
        }
}

// clopperPearsonLowerBound / UpperBound, include/state.h:134-151.
double orc_cp_lower(unsigned k, unsigned n, double alpha)
{
    if (k == 0)
        return 0.0;
    boost::math::beta_distribution<double> dist(k, n - k + 1);
    return boost::math::quantile(dist, alpha);
}

double orc_cp_upper(unsigned k, unsigned n, double alpha)
{
    if (k == n)
        return 1.0;
    boost::math::beta_distribution<double> dist(k + 1, n - k);
    return boost::math::quantile(dist, 1.0 - alpha);
}

// ---- PR-MPPI pieces -----------------------------------------------------------------------

int orc_pr_rollout(int prec, const dr_env_config* ec, const dr_prmppi_config* pc, const dr_sim_state* s0, const double* nom, const double* rob,
                   const float* noise, const int* thetas, uint64_t seed, uint64_t step, double* costNom, double* costRob)
{
    if (prec == 64)
        prRollout<double>(*ec, *pc, *s0, nom, rob, noise, thetas, seed, step, costNom, costRob);
    else
        prRollout<float>(*ec, *pc, *s0, nom, rob, noise, thetas, seed, step, costNom, costRob);
    return 0;
}

int orc_pr_update(int prec, const dr_prmppi_config* pc, double* costNom, double* costRob, const float* noise, const double* nom, const double* rob,
                  const float* invTemps, double* minCosts, double* cand1, double* cand2, double* newRob, double* nu, int blockorder)
{
    if (prec == 64)
        prUpdate<double>(*pc, costNom, costRob, noise, nom, rob, invTemps, minCosts, cand1, cand2, newRob, nu, blockorder);
    else
        prUpdate<float>(*pc, costNom, costRob, noise, nom, rob, invTemps, minCosts, cand1, cand2, newRob, nu, blockorder);
    return 0;
}

int orc_pr_candidates(int prec, const dr_env_config* ec, const dr_prmppi_config* pc, const dr_sim_state* s0, const double* cand1, const double* cand2,
                      const int* thetas, uint64_t seed, uint64_t step, int stream, double* fullCost, double* safeCost)
{
    if (prec == 64)
        prCandidates<double>(*ec, *pc, *s0, cand1, cand2, thetas, seed, step, (uint32_t)stream, fullCost, safeCost);
    else
        prCandidates<float>(*ec, *pc, *s0, cand1, cand2, thetas, seed, step, (uint32_t)stream, fullCost, safeCost);
    return 0;
}

// ---- environment step (engine dynStep, src/engine.cpp:286-312) -------------------------------

int orc_env_step(int prec, const dr_env_config* ec, int trueTheta, const float* action, dr_sim_state* state, float* belief, int updateBelief,
                 int considerBranching, float minConfidence, int loseOnOppWin, int applyNoise, uint64_t seed, uint64_t step, int t)
{
    auto run = [&](auto zero) -> int
    {
        using R = decltype(zero);
        Env<R> env(*ec);
        State<R> st = State<R>::from(*state);
        Branch<R> bs;
        R b0[DR_MAX_THETA];
        for (int th = 0; th < ec->n_theta; th++)
            b0[th] = belief[th];
        initBranchState(bs, b0, ec->n_theta, (R)minConfidence);
        StepFlags f{updateBelief != 0, considerBranching != 0, loseOnOppWin != 0, applyNoise != 0, true};
        EnvNoise rng(seed, 0u, 0u, step, S_ENV_STEP);
        rng.begin_step(0);
        R ego[DIM] = {(R)action[0], (R)action[1]};
        bool branched = false;
        int term = environmentStep(t, trueTheta, env, ego, f, st, bs, branched, (R)minConfidence, rng);
        st.to(*state);
        for (int th = 0; th < ec->n_theta; th++)
            belief[th] = (float)bs.belief[th];
        return term;
    };
    return prec == 64 ? run(0.0) : run(0.0f);
}

// Costs of a state (for unit tests): stateCost, PRMPPIstateCost, PRMPPIsafetyCost, finalCost.
void orc_costs(const dr_env_config* ec, const dr_mppi_config* mc, const dr_prmppi_config* pc, const dr_sim_state* s, float* out4)
{
    Env<float> env(*ec);
    State<float> st = State<float>::from(*s);
    MppiCosts<float> m = mppiCosts<float>(*mc);
    PrCosts<float> p = prCosts<float>(*pc);
    out4[0] = stateCost(st, env, m);
    out4[1] = prStateCost(st, env, p);
    out4[2] = prSafetyCost(st, env, p);
    out4[3] = finalCost(st, env, m.finalAdvWeight, m.finalOppAdvWeight);
}

} // extern "C"
