// rdst_options.h -- dictionary entries that select and parameterise the
// fully-coupled step, with the reference's names and defaults.
//
// Keys/defaults follow libraries/rhoDST/IOdictDST/IOdictDST.C:89-225
// (rhoDSTDict), the fvSchemes/fvSolution entries the step reads
// (tutorials/forwardStep/system/{fvSchemes,fvSolution}) and the thermo /
// transport coefficients of constant/thermophysicalProperties.  Selector
// names are those of the reference's run-time selection tables
// (newbaseFluxDST.C:64-84, JacobianDST.C:72-91, newIteration.C:59-78).
#pragma once

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace rdst {

enum FluxScheme { FLUX_KURGANOV = 0, FLUX_HLL, FLUX_HLLC, FLUX_HLLCP, FLUX_AUSMPLUS,
                  FLUX_AUSMPLUSUP, FLUX_AUSM };
enum Limiter { LIM_LINEAR = 0, LIM_UPWIND, LIM_OSPRE, LIM_VANLEER, LIM_MINMOD, LIM_VANALBADA,
               LIM_SUPERBEE, LIM_MUSCL, LIM_VENKATAKRISHNAN };
enum Solver { SOLVER_GMRES = 0, SOLVER_BICGSTAB, SOLVER_GAUSS_SEIDEL, SOLVER_ILU, SOLVER_AMG };
// ILU0: ILUC0 (exact ILU on the matrix pattern); CHOLESKY: the diagonal-only
// incomplete factorisation (D~ + L) D~^-1 (D~ + U); GAUSS_SEIDEL: forward
// block Gauss-Seidel sweeps (D + L)^-1; ILUCP: ILU on the pattern extended
// to cells within fillInLevel + 1 faces; AMG: one V-cycle of aggregation
// AMG with damped block-Jacobi smoothing
enum Precon { PRECON_NONE = 0, PRECON_DIAGONAL, PRECON_ILU0, PRECON_CHOLESKY, PRECON_GAUSS_SEIDEL, PRECON_ILUCP,
              PRECON_AMG };
enum Ddt { DDT_EULER = 0, DDT_STEADY, DDT_DUAL2ND };
enum Precision { PREC_FP64 = 0, PREC_FP32, PREC_BF16 };
enum Turbulence { TURB_LAMINAR = 0, TURB_SANEG, TURB_SARC1, TURB_SARC2, TURB_SA };

// preconditioners stored as incomplete block-LU factors (pivot inverses and
// L D~^-1 / U blocks on a row pattern)
inline bool lu_factored(Precon p) {
    return p == PRECON_ILU0 || p == PRECON_CHOLESKY || p == PRECON_GAUSS_SEIDEL || p == PRECON_ILUCP;
}

// Thrown by the parser; mapped to RDST_ERR_CONFIG / RDST_ERR_UNSUPPORTED.
struct ConfigError : std::runtime_error {
    bool unsupported;
    ConfigError(const std::string& m, bool u = false) : std::runtime_error(m), unsupported(u) {}
};

struct Options {
    // rhoDSTDict
    FluxScheme flux = FLUX_KURGANOV;
    bool flux_given = false;
    std::string jacobian = "Roe";
    bool dependent_W = true;          // dependentVariable W | deltaW
    double beta = 1.0;                // timeIntegration.beta
    bool dual = false;                // timeIntegration Dual (Dual.C:80-124)
    int max_inner_iter = 20;          // timeIntegration.maxInnerIter (IOdictDST.C:222-225)
    bool inner_correct_turbulence = false;   // timeIntegration.innerCorrectTurbulence
    int iteration_start = -1;         // residualControls.iterationStart (-1: 500 steady, 10 unsteady)
    double mag_converged_slope = 0.1; // residualControls.magConvergedSlope
    double min_residual = 1e-5;       // residualControls.minResudual
    bool adjust_time_step = true;     // timeControls.adjustTimeStep
    bool neighbouring = false;        // timeControls.neighbouring
    double initial_co = 1.0, min_co = 0.1, max_co = 50.0;
    bool direct_wave_speed = true;    // HLLC/HLLCP
    bool low_mach = false;            // AUSM+up
    double mainf = 0.5;               // AUSM+up
    double venkat_K = 5.0;            // Venkatakrishnan constant (not in the reference)
    bool frozen_turbulence = false;   // skip the turbulence update: mu_t held (not in the reference)
    // fvSchemes
    Ddt ddt = DDT_EULER;
    Limiter lim_rho = LIM_OSPRE, lim_U = LIM_OSPRE, lim_T = LIM_OSPRE;
    double grad_U_limit = 0.0;        // gradSchemes grad(U): 0 Gauss linear, k cellLimited Gauss linear k
    bool nut_linear_upwind = false;   // divSchemes div(phi,nuTilda): Gauss upwind | Gauss linearUpwind grad(nuTilda)
    // fvSolution: solvers.W
    Solver solver = SOLVER_BICGSTAB;
    Precon precon = PRECON_ILU0;
    int n_directions = 8;
    double tolerance = 1e-6, rel_tol = 0.0;
    int max_iter = 1000, min_iter = 0;
    int n_sweeps = 1;                 // Gauss-Seidel sweeps per application (nSweeps)
    int fill_in = 0;                  // ILUCp extension level (fillInLevel)
    int amg_pre = 0, amg_post = 2;    // AMG nPreSweeps / nPostSweeps (block-Jacobi sweeps per level)
    int amg_max_levels = 100;         // AMG nMaxLevels
    int amg_min_coarse = 4;           // AMG minCoarseEqns (cells on the coarsest level)
    int amg_coarsest_sweeps = 10;     // block-Jacobi sweeps on the coarsest level
    double amg_omega = 0.6;           // block-Jacobi damping of the AMG smoother
    // fvSolution: fieldBounds (updateFields.H:44-62)
    double rho_min = 1e-15, rho_max = 1e10, p_min = 1e-15, p_max = 1e10, T_min = 1e-15, T_max = 1e10;
    // thermophysicalProperties (perfectGas, hConstThermo, const/Sutherland transport)
    double R = 8314.47 / 28.9, Cp = 1004.5;
    double mu = 0.0, Pr = 1.0;        // constTransport
    double As = 0.0, Ts = 0.0;        // sutherlandTransport (As > 0 selects it)
    double Prt = 1.0;                 // turbulent Prandtl number (SAneg coeffDict default)
    Turbulence turbulence = TURB_LAMINAR;
    double nut_relax = 1.0;           // relaxationFactors.nuTilda
    int nut_sweeps = 10;              // point-Jacobi sweeps of the nuTilda system
    // time
    double delta_t = 1.0;             // controlDict deltaT (used when adjustTimeStep false)
    double start_time = 0.0;
    // B200 additions
    Precision precision = PREC_FP64;
    int basis32 = -1;                 // GMRES basis vectors in FP32 (-1: when precision is not fp64)
    int ilu_parts = 0;                // 0: choose from the mesh size; 1: exact global ILU(0)
    bool ilu_graph = false;           // subdomains by graph bisection (true) or coordinate bisection
    int ilu_order = -1;               // rows of a subdomain: 0 mesh order, 1 breadth-first (rdst_order.h),
                                      // -1 breadth-first with more than one subdomain, else mesh order
    bool ilu_bulk = true;             // ILU apply: task records, one bulk copy per task (same results)
    int ilu_factor_threads = 32;      // threads of the factorisation's CTA (one CTA per subdomain): 32, 64 or 128
    bool graphs = true;               // capture steps in CUDA graphs
    int device = -1;                  // GPU ordinal of the context (-1: the calling thread's current one)
    bool profile = false;             // event-time kernel classes inside steps

    double gamma() const { return Cp / (Cp - R); }
    double Cv() const { return Cp - R; }
};

inline std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\n;"), b = s.find_last_not_of(" \t\n;");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// runs of blanks -> one space (dictionary entries such as "Gauss  linear")
inline std::string collapse_ws(const std::string& s) {
    std::string out;
    bool sp = false;
    for (char ch : trim(s)) {
        if (ch == ' ' || ch == '\t' || ch == '\n') { sp = true; continue; }
        if (sp && !out.empty()) out += ' ';
        sp = false;
        out += ch;
    }
    return out;
}

inline bool parse_bool(const std::string& k, const std::string& v) {
    std::string t = trim(v);
    if (t == "true" || t == "yes" || t == "on" || t == "1") return true;
    if (t == "false" || t == "no" || t == "off" || t == "0") return false;
    throw ConfigError("option " + k + ": expected a bool, got '" + v + "'");
}

inline double parse_double(const std::string& k, const std::string& v) {
    std::string t = trim(v);
    char* end = nullptr;
    double d = std::strtod(t.c_str(), &end);
    if (t.empty() || *end != '\0' || !std::isfinite(d))
        throw ConfigError("option " + k + ": expected a number, got '" + v + "'");
    return d;
}

inline int parse_int(const std::string& k, const std::string& v) {
    double d = parse_double(k, v);
    if (d != std::floor(d)) throw ConfigError("option " + k + ": expected an integer");
    return (int)d;
}

inline void parse_pair(const std::string& k, const std::string& v, double& a, double& b) {
    std::istringstream is(v);
    std::string s1, s2;
    is >> s1 >> s2;
    a = parse_double(k, s1);
    b = parse_double(k, s2);
}

inline Limiter parse_limiter(const std::string& k, const std::string& v, bool vector) {
    std::string t = trim(v);
    if (t == "linear") return LIM_LINEAR;
    if (t == "upwind") return LIM_UPWIND;
    if (t == "Venkatakrishnan") return LIM_VENKATAKRISHNAN;
    // vector fields take the "V" (direction-aware) variants, scalars the plain ones
    std::string base = t;
    if (vector) {
        if (t.size() < 2 || t.back() != 'V')
            throw ConfigError("option " + k + ": vector reconstruction needs a V-limiter (e.g. OSPREV), got '" + t + "'", true);
        base = t.substr(0, t.size() - 1);
    }
    if (base == "OSPRE") return LIM_OSPRE;
    if (base == "vanLeer") return LIM_VANLEER;
    if (base == "Minmod") return LIM_MINMOD;
    if (base == "vanAlbada") return LIM_VANALBADA;
    if (base == "SuperBee") return LIM_SUPERBEE;
    if (base == "MUSCL") return LIM_MUSCL;
    throw ConfigError("option " + k + ": unknown interpolation scheme '" + t + "'");
}

inline FluxScheme parse_flux(const std::string& v) {
    std::string t = trim(v);
    if (t == "Kurganov") return FLUX_KURGANOV;
    if (t == "HLL") return FLUX_HLL;
    if (t == "HLLC") return FLUX_HLLC;
    if (t == "HLLCP") return FLUX_HLLCP;
    if (t == "AUSM+") return FLUX_AUSMPLUS;
    if (t == "AUSM+up") return FLUX_AUSMPLUSUP;
    if (t == "AUSM") return FLUX_AUSM;
    throw ConfigError("Unknown fluxScheme type " + t +
                      "\nValid fluxScheme types are: (AUSM AUSM+ AUSM+up HLL HLLC HLLCP Kurganov)");
}

inline Options parse_options(int n, const char* const* keys, const char* const* values) {
    Options o;
    std::map<std::string, std::string> kv;
    for (int i = 0; i < n; ++i) {
        if (!keys[i] || !values[i]) throw ConfigError("null option key/value");
        kv[trim(keys[i])] = values[i];
    }
    for (auto& it : kv) {
        const std::string& k = it.first;
        const std::string& v = it.second;
        std::string t = trim(v);
        if (k == "fluxScheme") { o.flux = parse_flux(v); o.flux_given = true; }
        else if (k == "Jacobian") {
            if (t != "Roe") throw ConfigError("Unknown Jacobian type " + t + "\nValid Jacobian types are: (Roe)");
            o.jacobian = t;
        }
        else if (k == "dependentVariable") {
            if (t == "W") o.dependent_W = true;
            else if (t == "deltaW") o.dependent_W = false;
            else throw ConfigError("dependentVariable must be W or deltaW");
        }
        else if (k == "timeIntegration.timeIntegration") {
            // GPU / GPUDual: the foam adapter's selector names for Single / Dual
            if (t == "Dual" || t == "GPUDual") o.dual = true;
            else if (t != "Single" && t != "GPU")
                throw ConfigError("Unknown timeIntegration type " + t + "\nValid timeIntegration types are: (Dual Single)");
        }
        else if (k == "timeIntegration.beta") o.beta = parse_double(k, v);
        else if (k == "timeIntegration.innerCorrectTurbulence") o.inner_correct_turbulence = parse_bool(k, v);
        else if (k == "timeIntegration.maxInnerIter") o.max_inner_iter = parse_int(k, v);
        else if (k == "timeControls.adjustTimeStep") o.adjust_time_step = parse_bool(k, v);
        else if (k == "timeControls.neighbouring") o.neighbouring = parse_bool(k, v);
        else if (k == "timeControls.initialCo") o.initial_co = parse_double(k, v);
        else if (k == "timeControls.minCo") o.min_co = parse_double(k, v);
        else if (k == "timeControls.maxCo") o.max_co = parse_double(k, v);
        else if (k == "residualControls.iterationStart") o.iteration_start = parse_int(k, v);
        else if (k == "residualControls.magConvergedSlope") o.mag_converged_slope = parse_double(k, v);
        else if (k == "residualControls.minResudual") o.min_residual = parse_double(k, v);
        else if (k.rfind("residualControls.", 0) == 0) {}
        else if (k == "directWaveSpeed") {
            o.direct_wave_speed = parse_bool(k, v);
            if (!o.direct_wave_speed)
                throw ConfigError("directWaveSpeed false leaves the HLLC wave speeds unset in the reference (HLLCDST.C:188-215); rejected", true);
        }
        else if (k == "lowMach") o.low_mach = parse_bool(k, v);
        else if (k == "Mainf") o.mainf = parse_double(k, v);
        else if (k == "addSpectralRadiusToPhysicalBoundaries") parse_bool(k, v);
        else if (k == "venkatakrishnanK") o.venkat_K = parse_double(k, v);
        else if (k == "frozenTurbulence") o.frozen_turbulence = parse_bool(k, v);
        else if (k == "ddtSchemes.default") {
            if (t == "Euler") o.ddt = DDT_EULER;
            else if (t == "steadyStateDST") o.ddt = DDT_STEADY;
            else if (t == "dual2ndDST") o.ddt = DDT_DUAL2ND;
            else throw ConfigError("Unknown ddtScheme " + t + "\nValid ddt schemes are: (Euler steadyStateDST dual2ndDST)");
        }
        else if (k == "interpolationSchemes.reconstruct(rho)") o.lim_rho = parse_limiter(k, v, false);
        else if (k == "interpolationSchemes.reconstruct(U)") o.lim_U = parse_limiter(k, v, true);
        else if (k == "interpolationSchemes.reconstruct(T)") o.lim_T = parse_limiter(k, v, false);
        else if (k == "solvers.W.solver") {
            // the asymmetric block-matrix solvers of Vector5typedefs.C:1655-1708
            if (t == "GMRES") o.solver = SOLVER_GMRES;
            else if (t == "BiCGStab") o.solver = SOLVER_BICGSTAB;
            else if (t == "GaussSeidel") o.solver = SOLVER_GAUSS_SEIDEL;
            else if (t == "ILU") o.solver = SOLVER_ILU;
            else if (t == "AMG") o.solver = SOLVER_AMG;
            else if (t == "CG")
                throw ConfigError("Unknown asymmetric matrix solver CG\n"
                                  "Valid asymmetric matrix solvers are: (AMG BiCGStab GMRES GaussSeidel ILU)");
            else throw ConfigError("Unknown block solver " + t + "\nValid solvers are: (AMG BiCGStab GMRES GaussSeidel ILU)");
        }
        else if (k == "solvers.W.preconditioner" || k == "solvers.W.preconditioner.preconditioner") {
            if (t == "ILUC0" || t == "ILU0") o.precon = PRECON_ILU0;
            else if (t == "Cholesky") o.precon = PRECON_CHOLESKY;
            else if (t == "GaussSeidel") o.precon = PRECON_GAUSS_SEIDEL;
            else if (t == "ILUCp") o.precon = PRECON_ILUCP;
            else if (t == "AMG") o.precon = PRECON_AMG;
            else if (t == "diagonal" || t == "Jacobi") o.precon = PRECON_DIAGONAL;
            else if (t == "none") o.precon = PRECON_NONE;
            else if (t == "SAMG")
                throw ConfigError("preconditioner " + t +
                                  " is not on this path (AMG Cholesky GaussSeidel ILUC0 ILUCp diagonal none)", true);
            else throw ConfigError("Unknown block preconditioner " + t);
        }
        else if (k == "solvers.W.nPreSweeps" || k == "solvers.W.preconditioner.nPreSweeps") o.amg_pre = parse_int(k, v);
        else if (k == "solvers.W.nPostSweeps" || k == "solvers.W.preconditioner.nPostSweeps") o.amg_post = parse_int(k, v);
        else if (k == "solvers.W.nMaxLevels" || k == "solvers.W.preconditioner.nMaxLevels")
            o.amg_max_levels = parse_int(k, v);
        else if (k == "solvers.W.minCoarseEqns" || k == "solvers.W.preconditioner.minCoarseEqns")
            o.amg_min_coarse = parse_int(k, v);
        else if (k == "solvers.W.smoother" || k == "solvers.W.preconditioner.smoother") {
            if (t != "Jacobi" && t != "diagonal")
                throw ConfigError("AMG smoother " + t + " is not on this path (Jacobi)", true);
        }
        else if (k == "amg.omega") o.amg_omega = parse_double(k, v);
        else if (k == "amg.coarsestSweeps") o.amg_coarsest_sweeps = parse_int(k, v);
        else if (k == "solvers.W.nSweeps" || k == "solvers.W.preconditioner.nSweeps") o.n_sweeps = parse_int(k, v);
        else if (k == "solvers.W.fillInLevel" || k == "solvers.W.preconditioner.fillInLevel") o.fill_in = parse_int(k, v);
        else if (k == "solvers.W.nDirections") o.n_directions = parse_int(k, v);
        else if (k == "solvers.W.tolerance") o.tolerance = parse_double(k, v);
        else if (k == "solvers.W.relTol") o.rel_tol = parse_double(k, v);
        else if (k == "solvers.W.maxIter") o.max_iter = parse_int(k, v);
        else if (k == "solvers.W.minIter") o.min_iter = parse_int(k, v);
        else if (k == "fieldBounds.rho") parse_pair(k, v, o.rho_min, o.rho_max);
        else if (k == "fieldBounds.p") parse_pair(k, v, o.p_min, o.p_max);
        else if (k == "fieldBounds.T") parse_pair(k, v, o.T_min, o.T_max);
        else if (k == "thermo.R") o.R = parse_double(k, v);
        else if (k == "thermo.Cp") o.Cp = parse_double(k, v);
        else if (k == "transport.mu") o.mu = parse_double(k, v);
        else if (k == "transport.Pr") o.Pr = parse_double(k, v);
        else if (k == "transport.As") o.As = parse_double(k, v);
        else if (k == "transport.Ts") o.Ts = parse_double(k, v);
        else if (k == "transport.Prt") o.Prt = parse_double(k, v);
        else if (k == "RASModel" || k == "turbulence") {
            if (t == "laminar") o.turbulence = TURB_LAMINAR;
            else if (t == "SAneg") o.turbulence = TURB_SANEG;
            else if (t == "SARC1") o.turbulence = TURB_SARC1;
            else if (t == "SARC2") o.turbulence = TURB_SARC2;
            // foam-extend's compressible SpalartAllmaras (the RAE2822 and
            // oneraM6Turb tutorials): the SARC equations without the
            // rotation/curvature multiplier (SARC1.C with
            // spalartShurCorrection false, SARC1.C:183-199)
            else if (t == "SpalartAllmaras") o.turbulence = TURB_SA;
            else throw ConfigError("Unknown RASModel " + t +
                                   "\nValid models are: (laminar SAneg SARC1 SARC2 SpalartAllmaras)");
        }
        else if (k == "relaxationFactors.nuTilda") o.nut_relax = parse_double(k, v);
        else if (k == "solvers.nuTilda.nSweeps") o.nut_sweeps = parse_int(k, v);
        else if (k == "controlDict.deltaT") o.delta_t = parse_double(k, v);
        else if (k == "controlDict.startTime") o.start_time = parse_double(k, v);
        else if (k == "precision") {
            if (t == "fp64") o.precision = PREC_FP64;
            else if (t == "fp32") o.precision = PREC_FP32;
            else if (t == "bf16") o.precision = PREC_BF16;
            else throw ConfigError("precision must be fp64, fp32 or bf16");
        }
        else if (k == "krylov.basis") {
            if (t == "fp64") o.basis32 = 0;
            else if (t == "fp32") o.basis32 = 1;
            else throw ConfigError("krylov.basis must be fp64 or fp32");
        }
        else if (k == "gradSchemes.default") {
            if (collapse_ws(t) != "Gauss linear")
                throw ConfigError("gradSchemes default " + t + " is not on this path (Gauss linear)", true);
        }
        else if (k == "gradSchemes.grad(U)") {
            // fvSchemes gradSchemes: Gauss linear, or cellLimited Gauss linear k
            const std::string g = collapse_ws(t);
            if (g == "Gauss linear") o.grad_U_limit = 0.0;
            else if (g.rfind("cellLimited Gauss linear ", 0) == 0) {
                o.grad_U_limit = parse_double(k, g.substr(25));
                if (!(o.grad_U_limit > 0.0 && o.grad_U_limit <= 1.0))
                    throw ConfigError("cellLimited coefficient must be in (0, 1]");
            } else throw ConfigError("gradSchemes grad(U) " + t + " is not on this path "
                                     "(Gauss linear, cellLimited Gauss linear k)", true);
        }
        else if (k == "divSchemes.div(phi,nuTilda)") {
            const std::string d = collapse_ws(t);
            if (d == "Gauss upwind") o.nut_linear_upwind = false;
            else if (d == "Gauss linearUpwind grad(nuTilda)") o.nut_linear_upwind = true;
            else throw ConfigError("divSchemes div(phi,nuTilda) " + t + " is not on this path "
                                   "(Gauss upwind, Gauss linearUpwind grad(nuTilda))", true);
        }
        else if (k == "divSchemes.div(tauMC)") {
            if (collapse_ws(t) != "Gauss linear")
                throw ConfigError("divSchemes div(tauMC) " + t + " is not on this path (Gauss linear)", true);
        }
        else if (k == "ilu.parts") o.ilu_parts = parse_int(k, v);
        else if (k == "ilu.bulk") o.ilu_bulk = parse_bool(k, v);
        else if (k == "ilu.factorThreads") {
            o.ilu_factor_threads = parse_int(k, v);
            if (o.ilu_factor_threads != 32 && o.ilu_factor_threads != 64 && o.ilu_factor_threads != 128)
                throw ConfigError("ilu.factorThreads must be 32, 64 or 128");
        }
        else if (k == "ilu.order") {
            if (t == "natural") o.ilu_order = 0;
            else if (t == "bfs") o.ilu_order = 1;
            else if (t == "auto") o.ilu_order = -1;
            else throw ConfigError("ilu.order must be natural, bfs or auto");
        }
        else if (k == "ilu.partition") {
            if (t == "rcb") o.ilu_graph = false;
            else if (t == "graph") o.ilu_graph = true;
            else throw ConfigError("ilu.partition must be rcb or graph");
        }
        else if (k == "graphs") o.graphs = parse_bool(k, v);
        else if (k == "device") o.device = parse_int(k, v);
        else if (k == "profile") o.profile = parse_bool(k, v);
        else throw ConfigError("unknown option '" + k + "'");
    }
    if (!o.flux_given) throw ConfigError("keyword fluxScheme is undefined in dictionary rhoDSTDict");
    if (o.basis32 < 0) o.basis32 = o.precision == PREC_FP64 ? 0 : 1;
    if (o.n_directions < 1 || o.n_directions > 64) throw ConfigError("solvers.W.nDirections must be in [1,64]");
    if (o.max_iter < 0 || o.min_iter < 0) throw ConfigError("solvers.W.maxIter/minIter must be >= 0");
    if (o.n_sweeps < 1 || o.n_sweeps > 64) throw ConfigError("solvers.W.nSweeps must be in [1,64]");
    if (o.fill_in < 0 || o.fill_in > 3) throw ConfigError("solvers.W.fillInLevel must be in [0,3]");
    // the stationary solvers iterate their own factorisation: Gauss-Seidel
    // sweeps, or (BlockILUSolver) the Cholesky-type incomplete factorisation
    if (o.solver == SOLVER_GAUSS_SEIDEL) o.precon = PRECON_GAUSS_SEIDEL;
    if (o.solver == SOLVER_ILU) o.precon = PRECON_CHOLESKY;
    if (o.solver == SOLVER_AMG) o.precon = PRECON_AMG;
    if (o.amg_pre < 0 || o.amg_post < 0 || o.amg_pre + o.amg_post < 1 || o.amg_pre > 16 || o.amg_post > 16)
        throw ConfigError("AMG nPreSweeps/nPostSweeps must be in [0,16] with at least one sweep");
    if (o.amg_max_levels < 2 || o.amg_min_coarse < 1 || o.amg_coarsest_sweeps < 1 || o.amg_coarsest_sweeps > 200)
        throw ConfigError("AMG needs nMaxLevels >= 2, minCoarseEqns >= 1, coarsestSweeps in [1,200]");
    if (!(o.amg_omega > 0.0 && o.amg_omega <= 1.0)) throw ConfigError("amg.omega must be in (0,1]");
    if (!(o.R > 0) || !(o.Cp > o.R)) throw ConfigError("thermo: need 0 < R < Cp");
    if (o.lim_U == LIM_VENKATAKRISHNAN) {}
    // dual-time stepping: the Dual iteration with the dual2ndDST ddt (the
    // pairing of the reference's dual-time tutorial), for the mean flow and
    // the nuTilda equation of every SA model (SARC1's strain-rate material
    // derivative with dual2ndDST's second-order ddt over the physical steps)
    if (o.dual != (o.ddt == DDT_DUAL2ND))
        throw ConfigError("timeIntegration Dual is restated with ddtSchemes dual2ndDST (and dual2ndDST with Dual)", true);
    if (o.iteration_start < 0) o.iteration_start = (o.ddt == DDT_STEADY) ? 500 : 10;
    if (o.max_inner_iter < 0) throw ConfigError("timeIntegration.maxInnerIter must be >= 0");
    return o;
}

// foam-extend scalar constants (double precision build)
constexpr double SMALL = 1.0e-15;
constexpr double VSMALL = 1.0e-300;
constexpr double SOLVER_SMALL = 1.0e-20;   // lduMatrix::small_ in normFactor

}  // namespace rdst
