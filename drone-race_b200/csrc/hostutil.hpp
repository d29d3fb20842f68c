// Host utilities shared by the C ABI translation units: error reporting, a device
// arena, conversion of the C-ABI configuration to the device layout, event timing.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/drmppi.h"
#include "instance.cuh"

namespace dr
{

std::string& lastError();

inline int fail(int code, const std::string& msg)
{
    lastError() = msg;
    return code;
}

#define CK(call)                                                                                                                                    \
    do                                                                                                                                              \
    {                                                                                                                                               \
        cudaError_t e_ = (call);                                                                                                                    \
        if (e_ != cudaSuccess)                                                                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? DR_ERR_OOM : DR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

inline size_t a16(size_t x)
{
    return (x + 15) & ~(size_t)15;
}
inline size_t a256(size_t x)
{
    return (x + 255) & ~(size_t)255;
}

// A device buffer that grows on demand (the prediction entry points' staging area).
struct DevScratch
{
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n)
    {
        if (n <= bytes)
            return cudaSuccess;
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess)
            bytes = n;
        return e;
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// Bump allocator over one cudaMalloc; every block is 256-byte aligned.
struct Arena
{
    std::vector<std::pair<void**, size_t>> req;
    void* base = nullptr;
    size_t total = 0;
    template <typename T> void add(T*& p, size_t bytes)
    {
        req.push_back({(void**)&p, bytes});
    }
    cudaError_t alloc()
    {
        size_t off = 0;
        for (auto& r : req)
            off = a256(off) + a256(std::max<size_t>(r.second, 16));
        total = off;
        cudaError_t e = cudaMalloc(&base, total);
        if (e != cudaSuccess)
            return e;
        cudaMemset(base, 0, total);
        off = 0;
        for (auto& r : req)
        {
            off = a256(off);
            *r.first = (char*)base + off;
            off += a256(std::max<size_t>(r.second, 16));
        }
        return cudaSuccess;
    }
    void release()
    {
        if (base)
            cudaFree(base);
        base = nullptr;
    }
};

inline EnvParams toEnvParams(const dr_env_config& c)
{
    EnvParams e{};
    e.dt = c.dt;
    e.droneRadius = c.drone_radius;
    e.posNoise = c.pos_noise_level;
    e.speedNoise = c.speed_noise_level;
    e.actionNoiseLevel = c.action_noise_level;
    for (int a = 0; a < 4; a++)
    {
        e.maxSpeed[a] = c.max_speed[a];
        e.maxAccel[a] = c.max_accel[a];
    }
    e.trackWidth = c.track_width;
    e.nWinLaps = c.n_win_laps;
    e.kP = c.kP;
    e.kV = c.kV;
    e.maxOppLatDistFact = c.max_opp_lat_dist_fact;
    e.trackLength = c.track_length;
    for (int th = 0; th < 8; th++)
        for (int o = 0; o < 3; o++)
        {
            e.s1[th][o] = c.opp_configs[th].s1[o];
            e.s2[th][o] = c.opp_configs[th].s2[o];
            e.s3[th][o] = c.opp_configs[th].s3[o];
            e.speedScale[th][o] = c.opp_configs[th].speed_scale[o];
            e.actionNoise[th][o] = c.opp_configs[th].action_noise[o];
        }
    return e;
}

// p[513][2] | t[513][2] | kappa[513] with the wrap-around sample appended.
// Certificate of the fast projection's local search (windowLocalSearch) for sample c of the
// centreline P ([NTS][2]): a squared radius r2 such that any point x with |x - q_c|^2 <= r2
// at which c is a local minimum of the squared distances f(j) = |x - q_j|^2 (f(c -+ 1) >=
// f(c) - EPS: what the search's truncated key comparisons establish) has f(k) > f(c) + EPS
// for every sample k with 2 <= |k - c| <= 2 WIN, so that c is the minimum of every window
// that holds it, by a margin far above the keys' resolution (2^-18 relative, at most 6e-5
// within the 4 m cap). In y = x - q_c with d_k = q_k - q_c, f(k) - f(c) = |d_k|^2 - 2 d_k.y:
// the points where sample k could win form the polygon
//   (-d_k).y <= (EPS - |d_k|^2) / 2,  d_{c-1}.y <= (|d_{c-1}|^2 + EPS) / 2,
//   d_{c+1}.y <= (|d_{c+1}|^2 + EPS) / 2,
// and the radius is the distance from y = 0 to the nearest of these polygons (their nearest
// point is the foot of 0 on an edge's line or a vertex that satisfies the other two), capped
// at 4 m (points farther from the centreline than that are outside every track). Stored
// shrunk by 1e-5 relative for the rounding of the kernel's distances.
inline float projectionCertificate(const float* P, int c)
{
    constexpr double EPS = 1e-3, CAP = 4.0;
    auto q = [&](int j, int d) { return (double)P[((j % NTS + NTS) % NTS) * 2 + d]; };
    auto vec = [&](int k, double* v) {
        v[0] = q(c + k, 0) - q(c, 0);
        v[1] = q(c + k, 1) - q(c, 1);
    };
    double dm[2], dp[2];
    vec(-1, dm);
    vec(1, dp);
    double r = CAP;
    for (int k = -2 * WIN; k <= 2 * WIN; k++)
    {
        if (k >= -1 && k <= 1)
            continue;
        double dk[2];
        vec(k, dk);
        const double n[3][2] = {{-dk[0], -dk[1]}, {dm[0], dm[1]}, {dp[0], dp[1]}};
        const double b[3] = {(EPS - (dk[0] * dk[0] + dk[1] * dk[1])) * 0.5, (dm[0] * dm[0] + dm[1] * dm[1] + EPS) * 0.5,
                             (dp[0] * dp[0] + dp[1] * dp[1] + EPS) * 0.5};
        auto feasible = [&](double y0, double y1) {
            for (int i = 0; i < 3; i++)
                if (n[i][0] * y0 + n[i][1] * y1 > b[i] + 1e-12 * (1.0 + std::fabs(b[i])))
                    return false;
            return true;
        };
        if (feasible(0.0, 0.0))
            return -1.0f; // sample k may win next to q_c itself: always scan
        double dist = INFINITY;
        for (int i = 0; i < 3; i++)
        {
            const double nn = n[i][0] * n[i][0] + n[i][1] * n[i][1];
            if (nn > 0.0)
            {
                const double y0 = n[i][0] * b[i] / nn, y1 = n[i][1] * b[i] / nn;
                if (feasible(y0, y1))
                    dist = std::min(dist, std::fabs(b[i]) / std::sqrt(nn));
            }
            for (int j = i + 1; j < 3; j++)
            {
                const double det = n[i][0] * n[j][1] - n[i][1] * n[j][0];
                if (std::fabs(det) <= 1e-18)
                    continue;
                const double y0 = (b[i] * n[j][1] - n[i][1] * b[j]) / det, y1 = (n[i][0] * b[j] - b[i] * n[j][0]) / det;
                if (feasible(y0, y1))
                    dist = std::min(dist, std::sqrt(y0 * y0 + y1 * y1));
            }
        }
        r = std::min(r, dist);
    }
    return r > 0.0 ? (float)(r * r * (1.0 - 1e-5)) : -1.0f;
}

inline std::vector<float> packGrids(const dr_env_config& c)
{
    std::vector<float> g(GRID_FLOATS, 0.0f);
    for (int i = -GRID_PAD; i < NTS + GRID_PAD; i++)
    {
        int k = (i + NTS) % NTS;
        g[GRID_P + i * 2] = c.p_grid[k * 2];
        g[GRID_P + i * 2 + 1] = c.p_grid[k * 2 + 1];
        g[GRID_PX + i] = c.p_grid[k * 2];
        g[GRID_PY + i] = c.p_grid[k * 2 + 1];
    }
    for (int i = 0; i <= NTS; i++)
    {
        int k = i % NTS;
        g[GRID_T + i * 2] = c.t_grid[k * 2];
        g[GRID_T + i * 2 + 1] = c.t_grid[k * 2 + 1];
        g[GRID_K + i] = c.kappa_grid[k];
    }
    for (int i = 0; i < NTS; i++)
        g[GRID_CERT + i] = projectionCertificate(c.p_grid, i);
    return g;
}

inline int checkEnv(const dr_env_config* env)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    if (env->n_opp < 1 || env->n_opp > DR_MAX_OPP || env->n_theta < 1 || env->n_theta > DR_MAX_THETA)
        return fail(DR_ERR_INVALID_ARG, "n_opp must be in [1,3] and n_theta in [1,8]");
    if (!env->p_grid || !env->t_grid || !env->kappa_grid)
        return fail(DR_ERR_INVALID_ARG, "track grids must be given");
    if (!(env->track_length > 0.0f) || !std::isfinite(env->track_length) || !(env->dt > 0.0f))
        return fail(DR_ERR_INVALID_ARG, "track_length and dt must be positive and finite");
    for (int i = 0; i < NTS; i++)
        if (!std::isfinite(env->p_grid[2 * i]) || !std::isfinite(env->p_grid[2 * i + 1]) || !std::isfinite(env->t_grid[2 * i]) ||
            !std::isfinite(env->t_grid[2 * i + 1]) || !std::isfinite(env->kappa_grid[i]))
            return fail(DR_ERR_INVALID_ARG, "track grids must be finite");
    return DR_OK;
}

// Gate race: validation of the C-ABI config (the reference checks the same counts
// against its compile-time sizes when it unpacks them, env_dronerace.cpp:156-219).
inline int checkGateEnv(const dr_gate_env_config* env)
{
    if (!env)
        return fail(DR_ERR_INVALID_ARG, "env is NULL");
    if (env->n_theta < 1 || env->n_theta > DR_MAX_THETA)
        return fail(DR_ERR_INVALID_ARG, "n_theta must be in [1,8]");
    if (env->n_gates < 1 || env->n_gates > DR_GATE_MAX_GATES)
        return fail(DR_ERR_INVALID_ARG, "n_gates must be in [1,16]");
    if (env->n_obstacles < 0 || env->n_obstacles > DR_GATE_MAX_OBSTACLES || env->n_round_obstacles < 0 ||
        env->n_round_obstacles > DR_GATE_MAX_OBSTACLES)
        return fail(DR_ERR_INVALID_ARG, "obstacle counts must be in [0,4]");
    if (env->i_mppi < 0 || env->i_mppi >= DR_GATE_AGENTS)
        return fail(DR_ERR_INVALID_ARG, "i_mppi must be 0 or 1");
    if (!env->track_points)
        return fail(DR_ERR_INVALID_ARG, "track_points must be given");
    if (!(env->dt > 0.0f) || !std::isfinite(env->dt))
        return fail(DR_ERR_INVALID_ARG, "dt must be positive and finite");
    for (int th = 0; th < env->n_theta; th++)
        if (env->opp_pid[th].raceline_index < 0 || env->opp_pid[th].raceline_index >= DR_GATE_RACELINES)
            return fail(DR_ERR_INVALID_ARG, "raceline_index must be 0 or 1");
    for (int i = 0; i < DR_GATE_RACELINES * NTS * 2; i++)
        if (!std::isfinite(env->track_points[i]))
            return fail(DR_ERR_INVALID_ARG, "track points must be finite");
    return DR_OK;
}

inline GateParams toGateParams(const dr_gate_env_config& c)
{
    GateParams g{};
    for (int d = 0; d < 2; d++)
    {
        g.arenaMin[d] = c.arena_min[d];
        g.arenaMax[d] = c.arena_max[d];
    }
    g.dt = c.dt;
    g.droneRadius = c.drone_radius;
    g.posNoise = c.pos_noise_level;
    g.speedNoise = c.speed_noise_level;
    g.actionNoiseLevel = c.action_noise_level;
    for (int a = 0; a < G_NA; a++)
    {
        g.maxSpeed[a] = c.max_speed[a];
        g.maxAccel[a] = c.max_accel[a];
    }
    g.nWinLaps = c.n_win_laps;
    g.targetDistance = c.target_distance;
    g.nGates = c.n_gates;
    g.nObs = c.n_obstacles;
    g.nRound = c.n_round_obstacles;
    g.iMppi = c.i_mppi;
    for (int i = 0; i < G_MAXG * 2; i++)
    {
        g.gateCenters[i] = c.gate_centers[i];
        g.gateVectors[i] = c.gate_vectors[i];
    }
    for (int i = 0; i < G_MAXG; i++)
        g.gateRadius[i] = c.gate_radius[i];
    for (int i = 0; i < G_MAXO * 4; i++)
        g.obstacles[i] = c.obstacles[i];
    for (int i = 0; i < G_MAXO * 2; i++)
        g.roundCenters[i] = c.round_obs_centers[i];
    for (int i = 0; i < G_MAXO; i++)
        g.roundRadius[i] = c.round_obs_radius[i];
    for (int th = 0; th < DR_MAX_THETA; th++)
    {
        const dr_pid_config& p = c.opp_pid[th];
        g.pidKp[th] = p.kp;
        g.pidKd[th] = p.kd;
        g.pidRepF[th] = p.repulsion_factor;
        g.pidRepP[th] = p.repulsion_power;
        g.pidRepD[th] = p.repulsion_dist_fact;
        g.pidRaceline[th] = p.raceline_index;
        g.pidNoise[th] = p.action_noise;
    }
    return g;
}

// racelines plus the sample the reference reads when s wraps to exactly 1.0f, then each
// raceline's padded x and y rows (the gate track buffer's layout, gate_model.cuh)
inline std::vector<float> packGateTrack(const dr_gate_env_config& c)
{
    std::vector<float> t(GATE_TRACK_FLOATS, 0.0f);
    const size_t n = (size_t)G_NR * NTS * 2;
    for (size_t i = 0; i < n; i++)
        t[i] = c.track_points[i];
    t[n] = c.track_points[(size_t)(G_NR - 1) * NTS * 2];
    t[n + 1] = c.track_points[(size_t)(G_NR - 1) * NTS * 2 + 1];
    for (int r = 0; r < G_NR; r++)
        for (int j = -G_RPAD; j < NTS + G_RPAD; j++)
        {
            const int src = ((j % NTS) + NTS) % NTS;
            const size_t row = (size_t)GATE_INTERLEAVED_FLOATS + (size_t)2 * r * G_ROW + G_RPAD + j;
            t[row] = c.track_points[((size_t)r * NTS + src) * 2];
            t[row + G_ROW] = c.track_points[((size_t)r * NTS + src) * 2 + 1];
        }
    for (int r = 0; r < G_NR; r++)
        for (int i = 0; i < NTS; i++)
            t[(size_t)GATE_CERT + (size_t)r * NTS + i] = projectionCertificate(c.track_points + (size_t)r * NTS * 2, i);
    return t;
}

inline int selectDevice(int device)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(DR_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n)
        return fail(DR_ERR_INVALID_ARG, "device index out of range");
    CK(cudaSetDevice(device));
    return DR_OK;
}

// buildSplineMatrix (src/mppi_controller.cu:56-141): natural cubic spline basis evaluated
// at t = 0..T-1, Thomas algorithm, endpoint hold, float arithmetic.
inline std::vector<float> splineMatrix(int T, int M, const int* knots)
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
            B[(size_t)t * M + basis] = val;
        }
    }
    return B;
}

inline int findConfidentHost(const float* belief, int nth, float threshold)
{
    for (int th = 0; th < nth; th++)
        if (belief[th] > threshold)
            return th + 1;
    return 0;
}

// Per-kernel device times from CUDA events recorded on the launching stream between
// the kernels of each step; averages over all steps recorded since reset().
struct Timer
{
    static constexpr int MAXM = 8;
    std::vector<std::string> names;
    std::vector<cudaEvent_t> ev;
    int steps = 0, cur = 0, nm = 0;
    std::vector<float> ms; // averages, filled by collect()
    void reset()
    {
        names.clear();
        ms.clear();
        steps = cur = nm = 0;
    }
    void begin()
    {
        cur = 0;
    }
    void mark(const char* name, cudaStream_t s)
    {
        size_t idx = (size_t)steps * MAXM + cur;
        while (ev.size() <= idx)
        {
            cudaEvent_t e;
            cudaEventCreate(&e);
            ev.push_back(e);
        }
        cudaEventRecord(ev[idx], s);
        if (steps == 0)
            names.push_back(name);
        cur++;
    }
    void end()
    {
        if (steps == 0)
            nm = cur;
        steps++;
    }
    void collect()
    {
        ms.assign(nm > 0 ? nm - 1 : 0, 0.0f);
        if (steps == 0 || nm < 2)
            return;
        cudaEventSynchronize(ev[(size_t)(steps - 1) * MAXM + nm - 1]);
        for (int j = 0; j + 1 < nm; j++)
        {
            double sum = 0.0;
            for (int s = 0; s < steps; s++)
            {
                float x = 0.0f;
                cudaEventElapsedTime(&x, ev[(size_t)s * MAXM + j], ev[(size_t)s * MAXM + j + 1]);
                sum += x;
            }
            ms[j] = (float)(sum / steps);
        }
    }
    // Times of this timer's marks after the first mark of `ref` in the same step (the
    // start of the step), averaged over the steps both timers recorded.
    std::vector<float> offsets(const Timer& ref) const
    {
        const int n = std::min(steps, ref.steps);
        std::vector<float> off(nm, 0.0f);
        if (n == 0 || ref.nm == 0)
            return off;
        cudaEventSynchronize(ev[(size_t)(steps - 1) * MAXM + nm - 1]);
        cudaEventSynchronize(ref.ev[(size_t)(ref.steps - 1) * MAXM + ref.nm - 1]);
        for (int j = 0; j < nm; j++)
        {
            double sum = 0.0;
            for (int s = 0; s < n; s++)
            {
                float x = 0.0f;
                cudaEventElapsedTime(&x, ref.ev[(size_t)s * MAXM], ev[(size_t)s * MAXM + j]);
                sum += x;
            }
            off[j] = (float)(sum / n);
        }
        return off;
    }
    ~Timer()
    {
        for (auto e : ev)
            cudaEventDestroy(e);
    }
};


// Averages of the recorded steps of a main-stream timer and, optionally, a side-stream
// timer; names point into the timers and stay valid until reset.
inline int kernelTimes(Timer& t, const char** names, float* ms, int n, int* count, Timer* side = nullptr)
{
    t.collect();
    if (side)
        side->collect();
    int c = 0;
    for (Timer* tm : {&t, side})
    {
        if (!tm)
            continue;
        for (size_t i = 0; i < tm->ms.size(); i++, c++)
            if (c < n)
            {
                if (names)
                    names[c] = tm->names[i].c_str();
                if (ms)
                    ms[c] = tm->ms[i];
            }
    }
    if (count)
        *count = c;
    return DR_OK;
}

// Start and end of every timed kernel after the start of the step (the main timer's
// first mark), averaged over the recorded steps: the schedule of the two streams.
inline int kernelTimeline(Timer& t, const char** names, float* start, float* end, int n, int* count, Timer* side = nullptr)
{
    int c = 0;
    for (Timer* tm : {&t, side})
    {
        if (!tm || tm->steps == 0)
            continue;
        const std::vector<float> off = tm->offsets(t);
        for (int j = 0; j + 1 < tm->nm; j++, c++)
            if (c < n)
            {
                if (names)
                    names[c] = tm->names[j].c_str();
                if (start)
                    start[c] = off[j];
                if (end)
                    end[c] = off[j + 1];
            }
    }
    if (count)
        *count = c;
    return DR_OK;
}

} // namespace dr
