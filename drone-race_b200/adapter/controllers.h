// Drop-in replacement for the reference's include/controllers.h.
//
// The public interface is the reference's, declaration for declaration
// (include/controllers.h:12-179): class names, constructors, getControl, and the public
// fields src/engine.cpp reads (h_belief, mppiConfig, h_nominal, failCount, epsilon,
// epsilonPartial, certifiedLoss, useNewPlan, h_nom_nominal, h_rob_nominal, resetNom,
// useNomPlan, min_nu, max_nu) -- so engine.cpp compiles unchanged. The private section,
// which held the reference's device buffers, is replaced by the handle of the C ABI in
// include/drmppi.h; the implementation is in controllers_drmppi.cpp.
#pragma once

#include "config.h"

#include <array>
#include <optional>
#include <vector>

#include "drmppi.h"

// The C-ABI environment the controllers hold: the strategic race's, or the gate race's
// when the reference is built with USE_ENV_DRONERACE (include/config.h:17-19).
#ifdef USE_ENV_DRONERACE
using DrAdapterEnv = dr_gate_env_config;
#else
using DrAdapterEnv = dr_env_config;
#endif

// forward
class SimulationEngine;

class Controller
{
  public:
    virtual ~Controller() = default;

    virtual void getControl(const SimState& state, float* outAction) = 0;

    SimulationEngine* engine = nullptr;
    std::array<float, N_TRUE_MODELS> h_belief; // host belief (nTrueModels). this is updated by the engine
};

class MPPIController : public Controller
{
  public:
    MPPIController() {};

    // if nominal (size (nModels+1) * T * dim) is not given, assumed 0
    MPPIController(const EnvironmentConfig& c, const MPPIConfig& mc, int s, std::optional<std::vector<float>> nominal = std::nullopt);

    ~MPPIController();

    void getControl(const SimState& state, float* outAction) override;

    MPPIConfig mppiConfig;

    std::vector<float> h_nominal; // host mirror (nBranchPlans, T, dim)

    std::vector<uint> failCountOld;
    std::vector<uint> failCountNew;
    std::vector<uint> failCount;
    double epsilonPartial;
    double epsilon;
    double certifiedLoss;
    bool useNewPlan;

    float min_nu = 0.0005f;
    float max_nu = 0.001f;

    std::vector<float> buildSplineMatrix();

  private:
    DrAdapterEnv envC{};
    dr_mppi_config cfgC{};
    std::vector<float> grids; // host copies of the track grids (p, dp, t, kappa) or of the racelines
    int seed = 0;
    dr_mppi* h = nullptr;
};

class PRMPPIController : public Controller
{
  public:
    PRMPPIController() {};

    PRMPPIController(const EnvironmentConfig& c, const PRMPPIConfig& mc, int s, std::optional<std::vector<float>> nominal = std::nullopt);

    ~PRMPPIController();

    void getControl(const SimState& state, float* outAction) override;

    PRMPPIConfig mppiConfig;

    std::vector<float> h_nom_nominal;
    std::vector<float> h_rob_nominal;

    bool resetNom;
    bool useNomPlan;

    float min_nu = 0.0005f;
    float max_nu = 0.001f;

  private:
    DrAdapterEnv envC{};
    dr_prmppi_config cfgC{};
    std::vector<float> grids;
    int seed = 0;
    dr_prmppi* h = nullptr;
};
