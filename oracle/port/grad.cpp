// TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// FP64 reference of the gradient path: the objective of an MPPI controller's noise-free
// rollout of its control sequence U (the reference's fullRolloutKernel, src/kernels.cu:
// 34-171, with every noise source off, averaged over the compatible hypotheses with the
// belief weights of aggregateBranchCostsKernel, kernels.cu:175-217), evaluated with the
// oracle's model (model.hpp, the restatement of env_stratrace.h / costs.cuh) on a
// forward-mode dual number: value and one directional derivative in double precision.
// The derivative along a direction (dU, dW) in control and cost-weight space is exact
// for the piecewise-smooth rollout with every discrete decision held; central finite
// differences of the value check it where no decision changes.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "model.hpp"

namespace orc
{

struct DD
{
    double v = 0, d = 0;
    DD() = default;
    DD(double x) : v(x) {}
    DD(float x) : v(x) {}
    DD(int x) : v(x) {}
    DD(double x, double dx) : v(x), d(dx) {}
    explicit operator double() const
    {
        return v;
    }
    explicit operator float() const
    {
        return (float)v;
    }
    explicit operator int() const
    {
        return (int)v;
    }
    DD& operator+=(DD o)
    {
        v += o.v;
        d += o.d;
        return *this;
    }
    DD& operator-=(DD o)
    {
        v -= o.v;
        d -= o.d;
        return *this;
    }
    DD& operator*=(DD o)
    {
        d = d * o.v + v * o.d;
        v *= o.v;
        return *this;
    }
    DD& operator/=(DD o)
    {
        const double q = v / o.v;
        d = (d - q * o.d) / o.v;
        v = q;
        return *this;
    }
};

inline DD operator+(DD a, DD b)
{
    return DD(a.v + b.v, a.d + b.d);
}
inline DD operator-(DD a, DD b)
{
    return DD(a.v - b.v, a.d - b.d);
}
inline DD operator*(DD a, DD b)
{
    return DD(a.v * b.v, a.d * b.v + a.v * b.d);
}
inline DD operator/(DD a, DD b)
{
    const double q = a.v / b.v;
    return DD(q, (a.d - q * b.d) / b.v);
}
inline DD operator-(DD a)
{
    return DD(-a.v, -a.d);
}
inline bool operator<(DD a, DD b)
{
    return a.v < b.v;
}
inline bool operator>(DD a, DD b)
{
    return a.v > b.v;
}
inline bool operator<=(DD a, DD b)
{
    return a.v <= b.v;
}
inline bool operator>=(DD a, DD b)
{
    return a.v >= b.v;
}
inline bool operator==(DD a, DD b)
{
    return a.v == b.v;
}
inline bool operator!=(DD a, DD b)
{
    return a.v != b.v;
}
inline DD sqrt(DD a)
{
    const double r = std::sqrt(a.v);
    return DD(r, r > 0 ? a.d / (2 * r) : 0.0);
}
inline DD exp(DD a)
{
    const double e = std::exp(a.v);
    return DD(e, a.d * e);
}
inline DD log(DD a)
{
    return DD(std::log(a.v), a.d / a.v);
}
inline DD fabs(DD a)
{
    return DD(std::fabs(a.v), a.v < 0 ? -a.d : a.d);
}
inline DD floor(DD a)
{
    return DD(std::floor(a.v), 0.0);
}
inline DD fmin(DD a, DD b)
{
    return a.v <= b.v ? a : b;
}
inline DD fmax(DD a, DD b)
{
    return a.v >= b.v ? a : b;
}
inline DD copysign(DD a, DD b)
{
    const double r = std::copysign(a.v, b.v);
    return DD(r, std::signbit(r) != std::signbit(a.v) ? -a.d : a.d);
}
inline DD pow(DD a, DD b)
{
    const double r = std::pow(a.v, b.v);
    double d = b.v * std::pow(a.v, b.v - 1) * a.d;
    if (b.d != 0)
        d += r * std::log(a.v) * b.d;
    return DD(r, d);
}
inline bool isfinite(DD a)
{
    return std::isfinite(a.v);
}
inline bool isinf(DD a)
{
    return std::isinf(a.v);
}

struct NoNoise
{
    void begin_step(uint32_t) {}
    float next()
    {
        return 0.0f;
    }
};

} // namespace orc

using namespace orc;

// out[0] = J, out[1] = dJ along (dU, dW). U: (n_theta+1) x M x 2 (M = n_knots in spline mode,
// n_timesteps in dense mode), B: the T x M spline basis (spline mode). w6: boundary_cost,
// outside_cost, win_cost, opp_win_cost, final_adv_weight, final_opp_adv_weight (NULL: mc's).
// dU / dW may be NULL (zero). sig (optional, n_theta x 3): steps rolled out, predTheta and
// branchingTime at the end, per hypothesis (-1 for an incompatible one).
extern "C" int orc_nominal_cost(const dr_env_config* ec, const dr_mppi_config* mc, const dr_sim_state* s0, const float* belief0, const float* B,
                                const double* U, const double* w6, const double* dU, const double* dW, double* out, int* sig)
{
    Env<DD> env(*ec);
    const int T = mc->n_timesteps, M = mc->use_splines ? mc->n_knots : T, nth = env.nth, nbp = nth + 1;
    const DD minConf = mc->min_confidence;
    double w[6] = {mc->boundary_cost, mc->outside_cost, mc->win_cost, mc->opp_win_cost, mc->final_adv_weight, mc->final_opp_adv_weight};
    if (w6)
        std::memcpy(w, w6, sizeof(w));
    auto wd = [&](int i) { return DD(w[i], dW ? dW[i] : 0.0); };
    MppiCosts<DD> cc{DD(mc->coll_dist_factor), wd(0), DD(mc->boundary_threshold_factor), wd(1), wd(2), wd(3), wd(4), wd(5)};
    std::vector<DD> u((size_t)nbp * M * 2);
    for (size_t i = 0; i < u.size(); i++)
        u[i] = DD(U[i], dU ? dU[i] : 0.0);
    DD initBelief[DR_MAX_THETA];
    for (int th = 0; th < nth; th++)
        initBelief[th] = belief0[th];
    Branch<DD> first;
    initBranchState(first, initBelief, nth, minConf);
    const StepFlags flags{true, true, true, false, true};
    DD num = 0.0, den = 0.0;
    for (int th = 0; th < nth; th++)
    {
        if (sig)
            sig[th * 3] = sig[th * 3 + 1] = sig[th * 3 + 2] = -1;
        if (!branchCompatibleWithModel(first.predTheta, th))
            continue;
        State<DD> st = State<DD>::from(*s0);
        Branch<DD> bs = first;
        DD cost = 0.0, decay = 1.0;
        bool stop = false;
        int tOrigin = 0, t = 0;
        NoNoise rng;
        for (; t < T && !stop; t++)
        {
            const int local = t - tOrigin, b = bs.predTheta;
            DD ego[DIM];
            for (int d = 0; d < DIM; d++)
            {
                if (mc->use_splines)
                {
                    DD sum = 0.0;
                    for (int m = 0; m < M; m++)
                        sum += DD((double)B[local * M + m]) * u[(size_t)(b * M + m) * 2 + d];
                    ego[d] = sum;
                }
                else
                    ego[d] = u[(size_t)(b * T + local) * 2 + d];
            }
            bool branched = false;
            const int term = environmentStep(t, th, env, ego, flags, st, bs, branched, minConf, rng);
            if (branched)
                tOrigin = t + 1;
            stop = term != TERM_NONE;
            cost += stateCost(st, env, cc) * decay;
            decay *= DD((double)DECAY);
        }
        cost += finalCost(st, env, cc.finalAdvWeight, cc.finalOppAdvWeight);
        if (sig)
        {
            sig[th * 3] = t;
            sig[th * 3 + 1] = bs.predTheta;
            sig[th * 3 + 2] = bs.branchingTime;
        }
        if (!std::isfinite(cost.v))
            continue;
        num += DD((double)belief0[th]) * cost;
        den += DD((double)belief0[th]);
    }
    if (den.v > 1e-30)
    {
        const DD J = num / den;
        out[0] = J.v;
        out[1] = J.d;
    }
    else
    {
        out[0] = INFINITY;
        out[1] = 0.0;
    }
    return 0;
}
