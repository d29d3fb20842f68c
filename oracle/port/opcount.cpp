// TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// Algorithmic work of one environment step, measured by running the oracle's model
// (model.hpp, the restatement of env_stratrace.h / costs.cuh) with an operation-counting
// scalar. Every floating-point operation is counted once: add/sub, mul, div, sqrt, exp,
// log, pow, min/max/abs/floor/copysign; comparisons are counted separately and are not
// FLOPs. With `dedup` = 1, an operation whose opcode and operands were already seen in
// the same environment step is not counted again: the work of an implementation that
// evaluates each distinct expression once per step (the reference re-evaluates some
// track quantities several times per step; the CUDA kernels share them). With `dedup` = 2
// an operation is counted once per step index over all the samples counted: the work of an
// implementation that also shares what samples have in common at the same step (the
// verification's ego moves, identical for samples that took the same branch at the same
// step when the ego draws no noise). `dedup | 4` also leaves out work whose result nothing
// reads: once a sample has committed to a branch, its belief update and the other
// hypotheses' opponent actions (the kernels skip them; the reference does them).
// `dedup | 8` counts the projections' searches as the kernels run them where their
// certificate holds (SearchCount in model.hpp: the local search of the window, the gate
// race's walks without their margin scans), the results still taken from the searches
// as the reference writes them.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_set>
#include <vector>

#include "gate_model.hpp"
#include "model.hpp"

namespace orc
{

struct OpStats
{
    double add = 0, mul = 0, div = 0, sqrt_ = 0, exp_ = 0, log_ = 0, pow_ = 0, minmax = 0, cmp = 0;
};

struct CountCtx
{
    OpStats s;
    bool dedup = false;
    std::unordered_set<uint64_t> seen;
    std::vector<std::unordered_set<uint64_t>> seenAt; // dedup 2: per step index
};

inline thread_local CountCtx* g_ctx = nullptr;
inline thread_local CountCtx* g_paused = nullptr;

// SearchCount::pause: suspends counting (on) and resumes it (off)
inline void pauseCounting(bool on)
{
    if (on)
    {
        g_paused = g_ctx;
        g_ctx = nullptr;
    }
    else if (g_paused)
    {
        g_ctx = g_paused;
        g_paused = nullptr;
    }
}

// sets SearchCount for one counting call and clears it on every return path
struct SearchCountScope
{
    explicit SearchCountScope(bool local)
    {
        g_searchCount.local = local;
        g_searchCount.pause = pauseCounting;
    }
    ~SearchCountScope()
    {
        g_searchCount.local = false;
        g_paused = nullptr;
    }
};

inline uint64_t dbits(double x)
{
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
}

inline bool fresh(int op, double a, double b, bool commutative)
{
    if (!g_ctx)
        return false;
    if (!g_ctx->dedup)
        return true;
    uint64_t x = dbits(a), y = dbits(b);
    if (commutative && x > y)
        std::swap(x, y);
    uint64_t h = (uint64_t)op * 0x9E3779B97F4A7C15ull;
    h ^= x + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
    h ^= y + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
    return g_ctx->seen.insert(h).second;
}

struct CF
{
    double v = 0;
    CF() = default;
    CF(double x) : v(x) {}
    CF(float x) : v(x) {}
    CF(int x) : v(x) {}
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
    CF& operator+=(CF o);
    CF& operator-=(CF o);
    CF& operator*=(CF o);
    CF& operator/=(CF o);
};

#define CF_BIN(opname, expr, field, op, comm)                                                                                                         \
    inline CF opname(CF a, CF b)                                                                                                                    \
    {                                                                                                                                               \
        if (fresh(op, a.v, b.v, comm))                                                                                                              \
            g_ctx->s.field += 1;                                                                                                                    \
        return CF(expr);                                                                                                                            \
    }
CF_BIN(operator+, a.v + b.v, add, 1, true)
CF_BIN(operator-, a.v - b.v, add, 2, false)
CF_BIN(operator*, a.v * b.v, mul, 3, true)
CF_BIN(operator/, a.v / b.v, div, 4, false)
#undef CF_BIN

inline CF& CF::operator+=(CF o)
{
    *this = *this + o;
    return *this;
}
inline CF& CF::operator-=(CF o)
{
    *this = *this - o;
    return *this;
}
inline CF& CF::operator*=(CF o)
{
    *this = *this * o;
    return *this;
}
inline CF& CF::operator/=(CF o)
{
    *this = *this / o;
    return *this;
}
inline CF operator-(CF a)
{
    return CF(-a.v);
}

#define CF_CMP(opname, expr)                                                                                                                          \
    inline bool opname(CF a, CF b)                                                                                                                  \
    {                                                                                                                                               \
        if (g_ctx)                                                                                                                                  \
            g_ctx->s.cmp += 1;                                                                                                                      \
        return expr;                                                                                                                                \
    }
CF_CMP(operator<, a.v < b.v)
CF_CMP(operator>, a.v > b.v)
CF_CMP(operator<=, a.v <= b.v)
CF_CMP(operator>=, a.v >= b.v)
CF_CMP(operator==, a.v == b.v)
CF_CMP(operator!=, a.v != b.v)
#undef CF_CMP

#define CF_UN(fname, expr, field, op)                                                                                                                 \
    inline CF fname(CF a)                                                                                                                           \
    {                                                                                                                                               \
        if (fresh(op, a.v, 0.0, false))                                                                                                             \
            g_ctx->s.field += 1;                                                                                                                    \
        return CF(expr);                                                                                                                            \
    }
CF_UN(sqrt, std::sqrt(a.v), sqrt_, 10)
CF_UN(exp, std::exp(a.v), exp_, 11)
CF_UN(log, std::log(a.v), log_, 12)
CF_UN(fabs, std::fabs(a.v), minmax, 13)
CF_UN(floor, std::floor(a.v), minmax, 14)
#undef CF_UN

inline CF fmin(CF a, CF b)
{
    if (fresh(20, a.v, b.v, true))
        g_ctx->s.minmax += 1;
    return CF(std::fmin(a.v, b.v));
}
inline CF fmax(CF a, CF b)
{
    if (fresh(21, a.v, b.v, true))
        g_ctx->s.minmax += 1;
    return CF(std::fmax(a.v, b.v));
}
inline CF copysign(CF a, CF b)
{
    if (fresh(22, a.v, b.v, false))
        g_ctx->s.minmax += 1;
    return CF(std::copysign(a.v, b.v));
}
inline CF pow(CF a, CF b)
{
    if (fresh(23, a.v, b.v, false))
        g_ctx->s.pow_ += 1;
    return CF(std::pow(a.v, b.v));
}
inline bool isfinite(CF a)
{
    return std::isfinite(a.v);
}
inline bool isinf(CF a)
{
    return std::isinf(a.v);
}

} // namespace orc

using namespace orc;

// out[0..8] = add, mul, div, sqrt, exp, log, pow, minmax, cmp; out[9] = environment steps.
// kind 0: MPPI rollout of `nsamples` samples (dense controls, nominal + noise inputs);
// kind 1: verification rollouts of `nsamples` samples of the dense plan `nominal`.
// the counting loop for either model (model.hpp / gate_model.hpp, found by argument-
// dependent lookup); makeFlags(kind) gives the environmentStep flags of the rollout
// (kind 0) or the verification (kind 1)
template <typename EnvT, typename StateT, typename S0, typename MakeFlags>
static int countOps(const EnvT& env, const dr_mppi_config* mc, const S0* s0, const float* belief0, const float* nominal, const float* noise,
                    uint64_t seed, uint64_t step, int nsamples, int kind, int dedup, double* out, MakeFlags makeFlags)
{
    // dedup | 4: skip the work whose result nothing reads (the belief update and the other
    // hypotheses' actions once a sample has committed to a branch), as the kernels do
    const bool skipDead = (dedup & 4) != 0;
    const SearchCountScope searches((dedup & 8) != 0);
    dedup &= 3;
    CountCtx ctx;
    ctx.dedup = dedup != 0;
    if (dedup == 2)
        ctx.seenAt.resize((size_t)std::max(mc->n_timesteps, mc->verif_horizon) + 1);
    const int K = mc->n_samples, T = mc->n_timesteps, nth = env.nth;
    const CF minConf = mc->min_confidence;
    MppiCosts<CF> cc{mc->coll_dist_factor, mc->boundary_cost, mc->boundary_threshold_factor, mc->outside_cost,
                     mc->win_cost,         mc->opp_win_cost, mc->final_adv_weight,          mc->final_opp_adv_weight};
    CF initBelief[DR_MAX_THETA];
    for (int th = 0; th < nth; th++)
        initBelief[th] = belief0[th];
    double steps = 0;
    const Key key(seed);
    for (int s = 0; s < nsamples && s < (kind == 0 ? K : mc->n_verif_samples); s++)
    {
        Branch<CF> first;
        initBranchState(first, initBelief, nth, minConf);
        int th0 = 0, th1 = nth;
        int thetaV = 0;
        if (kind == 1)
        {
            float u = uniform_from_word(draw(key, (uint32_t)s, 0u, step, S_VERIF_THETA, 0).v[0]);
            float cdf = 0.0f;
            thetaV = nth - 1;
            for (int k = 0; k < nth; k++)
            {
                cdf += belief0[k];
                if (u <= cdf)
                {
                    thetaV = k;
                    break;
                }
            }
            th0 = 0;
            th1 = 1;
        }
        for (int th = th0; th < th1; th++)
        {
            int theta = kind == 1 ? thetaV : th;
            if (kind == 0 && !branchCompatibleWithModel(first.predTheta, theta))
                continue;
            StateT st = StateT::from(*s0);
            Branch<CF> bs = first;
            CF cost = 0.0, decay = 1.0;
            bool stop = false;
            int tOrigin = 0;
            EnvNoise rng(seed, (uint32_t)s, kind == 0 ? ((uint32_t)theta << 16) : 0u, step, kind == 0 ? S_MPPI_ROLL_ENV : S_VERIF_ENV);
            auto flags = makeFlags(kind);
            flags.skipDeadBelief = skipDead;
            int H = kind == 0 ? T : mc->verif_horizon;
            for (int t = 0; t < H && !stop; t++)
            {
                if (dedup == 2)
                    std::swap(ctx.seen, ctx.seenAt[t]); // the set of step t over the samples so far
                else
                    ctx.seen.clear();
                g_ctx = nullptr;
                rng.begin_step((uint32_t)t);
                int local = t - tOrigin;
                int b = bs.predTheta;
                g_ctx = &ctx;
                CF ego[DIM];
                for (int d = 0; d < DIM; d++)
                {
                    CF nom = nominal[(b * T + local) * DIM + d];
                    if (kind == 0)
                        ego[d] = nom + CF(noise[((size_t)(b * T + local) * K + s) * DIM + d]);
                    else
                        ego[d] = nom;
                }
                bool branched = false;
                int term = environmentStep(t, theta, env, ego, flags, st, bs, branched, minConf, rng);
                if (branched)
                    tOrigin = t + 1;
                stop = (term != TERM_NONE);
                if (kind == 0)
                {
                    cost += stateCost(st, env, cc) * decay;
                    decay *= CF(DECAY);
                }
                else if (term == TERM_LOSE || term == TERM_WIN || term == TERM_OPP_WIN)
                    stop = true;
                g_ctx = nullptr;
                if (dedup == 2)
                    std::swap(ctx.seen, ctx.seenAt[t]);
                steps += 1;
            }
        }
    }
    g_ctx = nullptr;
    const OpStats& o = ctx.s;
    double v[10] = {o.add, o.mul, o.div, o.sqrt_, o.exp_, o.log_, o.pow_, o.minmax, o.cmp, steps};
    std::memcpy(out, v, sizeof(v));
    return 0;
}

extern "C" int orc_count_ops(const dr_env_config* ec, const dr_mppi_config* mc, const dr_sim_state* s0, const float* belief0, const float* nominal,
                             const float* noise, uint64_t seed, uint64_t step, int nsamples, int kind, int dedup, double* out)
{
    Env<CF> env(*ec);
    return countOps<Env<CF>, State<CF>>(env, mc, s0, belief0, nominal, noise, seed, step, nsamples, kind, dedup, out,
                                        [](int k) { return StepFlags{true, true, k == 0, true, true}; });
}

// the same on the gate race (gate_model.hpp): environmentStep<true, true, false, k == 0>
extern "C" int orc_gate_count_ops(const dr_gate_env_config* ec, const dr_mppi_config* mc, const dr_gate_state* s0, const float* belief0,
                                  const float* nominal, const float* noise, uint64_t seed, uint64_t step, int nsamples, int kind, int dedup, double* out)
{
    gate::Env<CF> env(*ec);
    const float margin = mc->gate_traversal_margin;
    return countOps<gate::Env<CF>, gate::State<CF>>(env, mc, s0, belief0, nominal, noise, seed, step, nsamples, kind, dedup, out,
                                                    [margin](int k) { return gate::Flags{true, true, false, k == 0, true, margin}; });
}

// The PR-MPPI rollout step (PRMPPIfullRolloutKernel, prmppi_kernels.cu:55-130):
// environmentStep<false, false, true> under one sampled hypothesis, PRMPPIstateCost and
// PRMPPIsafetyCost each step. out as orc_count_ops; nsamples samples of the nominal
// controls plus noise [T][K][2] under hypothesis `theta`.
extern "C" int orc_pr_count_ops(const dr_env_config* ec, const dr_prmppi_config* pc, const dr_sim_state* s0, const float* nominal, const float* noise,
                                int theta, uint64_t seed, uint64_t step, int nsamples, int dedup, double* out)
{
    Env<CF> env(*ec);
    const SearchCountScope searches((dedup & 8) != 0);
    dedup &= 3;
    CountCtx ctx;
    ctx.dedup = dedup != 0;
    const int K = pc->n_samples, T = pc->n_timesteps;
    PrCosts<CF> cc{pc->coll_dist_factor, pc->boundary_cost, pc->boundary_threshold_factor, pc->win_cost,
                   pc->opp_win_cost,     pc->final_adv_weight, pc->final_opp_adv_weight, pc->safety_weight};
    const StepFlags flags{false, false, true, true, false};
    double steps = 0;
    for (int s = 0; s < nsamples && s < K; s++)
    {
        State<CF> st = State<CF>::from(*s0);
        Branch<CF> bs{};
        CF running = 0.0, safe = -INFINITY, decay = 1.0;
        bool stop = false;
        EnvNoise rng(seed, (uint32_t)s, 0u, step, S_PR_ROLL_ENV);
        for (int t = 0; t < T && !stop; t++)
        {
            ctx.seen.clear();
            g_ctx = nullptr;
            rng.begin_step((uint32_t)t);
            g_ctx = &ctx;
            CF ego[DIM];
            for (int d = 0; d < DIM; d++)
                ego[d] = CF(nominal[t * DIM + d]) + CF(noise[((size_t)t * K + s) * DIM + d]);
            bool branched = false;
            int term = environmentStep(t, theta, env, ego, flags, st, bs, branched, CF(0.0), rng);
            stop = (term != TERM_NONE);
            running += decay * prStateCost(st, env, cc);
            safe = fmax(safe, prSafetyCost(st, env, cc));
            decay *= CF(DECAY);
            g_ctx = nullptr;
            steps += 1;
        }
    }
    g_ctx = nullptr;
    const OpStats& o = ctx.s;
    double v[10] = {o.add, o.mul, o.div, o.sqrt_, o.exp_, o.log_, o.pow_, o.minmax, o.cmp, steps};
    std::memcpy(out, v, sizeof(v));
    return 0;
}
