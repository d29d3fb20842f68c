// Track preprocessing on the device: the StratRace track grids of the reference's Python
// front-end (python-src/utils.py:390-427) for many tracks at once, one CTA per track.
//
//   the closed curve, sampled at 512 points q_k (the caller evaluates its track function),
//   is re-parametrised by the cumulative chord length s_k (s_0 = 0, s_512 = L); x(s) and
//   y(s) are periodic cubic splines through (s_k, q_k) (scipy CubicSpline with
//   bc_type="periodic" in the reference); the grids are their values, first and second
//   derivatives at s = k L / 512: p, dp, the unit tangent t = dp / max(|dp|, 1e-6) and the
//   curvature (x'y'' - y'x'') / max((x'^2 + y'^2)^1.5, 1e-6), rounded to float32 as the wire
//   format carries them.
//
// The spline's slopes solve the cyclic tridiagonal system of C2 continuity,
//   h_i m_{i-1} + 2 (h_{i-1} + h_i) m_i + h_{i-1} m_{i+1} = 3 (h_i d_{i-1} + h_{i-1} d_i),
// with h_i = s_{i+1} - s_i and d_i = (y_{i+1} - y_i) / h_i, indices modulo 512; it is solved
// in double precision by the Thomas algorithm with a Sherman-Morrison correction for the
// two corner entries (one thread, both coordinates). Each grid point is then a cubic Hermite
// evaluation on its interval (found by binary search), one thread per point.
#include <cstdio>

#include "../../include/drmppi.h"
#include "launch.h"

namespace dr
{

namespace
{
constexpr int NT = DR_N_TRACK_SAMPLES;

// Solves the cyclic system a_i m_{i-1} + b_i m_i + c_i m_{i+1} = r_i (i mod NT) for the two
// right-hand sides r[0], r[1] in place, with a_i = h_i, b_i = 2 (h_{i-1} + h_i),
// c_i = h_{i-1}: Sherman-Morrison over the Thomas algorithm (u = (gamma, 0, .., 0, c_{NT-1}),
// v = (1, 0, .., 0, a_0 / gamma)). `w` and `z` are scratch of NT entries.
__device__ void cyclicSolve(const double* h, double (*r)[NT], double* w, double* z)
{
    auto A = [&](int i) { return h[i]; };
    auto Cc = [&](int i) { return h[(i + NT - 1) % NT]; };
    auto Bd = [&](int i) { return 2.0 * (h[(i + NT - 1) % NT] + h[i]); };
    const double gamma = -Bd(0);
    // T' = T - u v^T has diagonal b_0 - gamma and b_{NT-1} - a_0 c_{NT-1} / gamma
    auto diag = [&](int i) { return i == 0 ? Bd(0) - gamma : (i == NT - 1 ? Bd(NT - 1) - A(0) * Cc(NT - 1) / gamma : Bd(i)); };
    double beta = diag(0);
    w[0] = Cc(0) / beta;
    r[0][0] /= beta;
    r[1][0] /= beta;
    z[0] = gamma / beta;
    for (int i = 1; i < NT; i++)
    {
        beta = diag(i) - A(i) * w[i - 1];
        const double ui = i == NT - 1 ? Cc(NT - 1) : 0.0;
        w[i] = Cc(i) / beta;
        r[0][i] = (r[0][i] - A(i) * r[0][i - 1]) / beta;
        r[1][i] = (r[1][i] - A(i) * r[1][i - 1]) / beta;
        z[i] = (ui - A(i) * z[i - 1]) / beta;
    }
    for (int i = NT - 2; i >= 0; i--)
    {
        r[0][i] -= w[i] * r[0][i + 1];
        r[1][i] -= w[i] * r[1][i + 1];
        z[i] -= w[i] * z[i + 1];
    }
    const double g = A(0) / gamma;
    const double vz = z[0] + g * z[NT - 1];
    const double f0 = (r[0][0] + g * r[0][NT - 1]) / (1.0 + vz);
    const double f1 = (r[1][0] + g * r[1][NT - 1]) / (1.0 + vz);
    for (int i = 0; i < NT; i++)
    {
        r[0][i] -= f0 * z[i];
        r[1][i] -= f1 * z[i];
    }
}
} // namespace

__global__ void __launch_bounds__(NT) track_grids_kernel(const double* __restrict__ q, float* __restrict__ out, float* __restrict__ lengths)
{
    __shared__ double sq[NT + 1][2];
    __shared__ double s[NT + 1];
    __shared__ double h[NT];
    __shared__ double m[2][NT];
    __shared__ double w[NT], z[NT];
    const int tr = blockIdx.x, k = threadIdx.x;
    const double* qt = q + (size_t)tr * NT * 2;
    sq[k][0] = qt[k * 2];
    sq[k][1] = qt[k * 2 + 1];
    if (k == 0)
    {
        sq[NT][0] = qt[0];
        sq[NT][1] = qt[1];
    }
    __syncthreads();
    // chord lengths and their running sum, in sample order (numpy's cumsum)
    if (k == 0)
    {
        s[0] = 0.0;
        for (int i = 0; i < NT; i++)
        {
            const double dx = sq[i + 1][0] - sq[i][0], dy = sq[i + 1][1] - sq[i][1];
            s[i + 1] = s[i] + sqrt(dx * dx + dy * dy);
        }
    }
    __syncthreads();
    h[k] = s[k + 1] - s[k];
    __syncthreads();
    // cyclic system of the slopes (one matrix, a right-hand side per coordinate)
    const int km = (k + NT - 1) % NT;
    for (int d = 0; d < 2; d++)
    {
        const double dPrev = (sq[k][d] - sq[km][d]) / h[km];
        const double dCur = (sq[k + 1][d] - sq[k][d]) / h[k];
        m[d][k] = 3.0 * (h[k] * dPrev + h[km] * dCur);
    }
    __syncthreads();
    if (k == 0)
        cyclicSolve(h, m, w, z);
    __syncthreads();
    const double L = s[NT];
    const double sg = (double)k * (L / NT); // numpy linspace(0, L, 512, endpoint=False)
    // interval: the last knot <= sg (searchsorted right, minus one), within [0, NT - 1]
    int lo = 0, hi = NT;
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (s[mid] <= sg)
            lo = mid;
        else
            hi = mid;
    }
    const int i = lo;
    const double t = sg - s[i], hh = h[i];
    double v[2], d1[2], d2[2];
    for (int d = 0; d < 2; d++)
    {
        const double slope = (sq[i + 1][d] - sq[i][d]) / hh;
        const double m0 = m[d][i], m1 = m[d][(i + 1) % NT];
        const double c2 = (3.0 * slope - 2.0 * m0 - m1) / hh;
        const double c3 = (m0 + m1 - 2.0 * slope) / (hh * hh);
        v[d] = sq[i][d] + t * (m0 + t * (c2 + t * c3));
        d1[d] = m0 + t * (2.0 * c2 + 3.0 * c3 * t);
        d2[d] = 2.0 * c2 + 6.0 * c3 * t;
    }
    const double nrm = sqrt(d1[0] * d1[0] + d1[1] * d1[1]);
    const double den = fmax(nrm, 1e-6);
    const double kap = (d1[0] * d2[1] - d1[1] * d2[0]) / fmax(pow(d1[0] * d1[0] + d1[1] * d1[1], 1.5), 1e-6);
    float* o = out + (size_t)tr * (NT * 7);
    o[k * 2] = (float)v[0];
    o[k * 2 + 1] = (float)v[1];
    o[NT * 2 + k * 2] = (float)d1[0];
    o[NT * 2 + k * 2 + 1] = (float)d1[1];
    o[NT * 4 + k * 2] = (float)(d1[0] / den);
    o[NT * 4 + k * 2 + 1] = (float)(d1[1] / den);
    o[NT * 6 + k] = (float)kap;
    if (k == 0)
        lengths[tr] = (float)L;
}

cudaError_t launchTrackGrids(cudaStream_t stream, const double* q, int nTracks, float* out, float* lengths)
{
    track_grids_kernel<<<nTracks, NT, 0, stream>>>(q, out, lengths);
    return cudaGetLastError();
}

} // namespace dr
