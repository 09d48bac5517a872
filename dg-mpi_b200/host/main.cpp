// main.cpp -- dg_solve: the reference's driver (src/exec/main.cpp +
// src/post/main.cpp) on the B200 path.  It keeps the reference's TOML deck,
// its Solver / StepperBase / take_time_step structure and its post-processing
// L2 error, and calls libdg_b200.so through the C ABI for the hot path.
//
//   dg_solve [-input input.toml] [-check]     (default deck: input.toml)
//   dg_solve [-input input.toml] -post [data.h5]
//            the reference's post tool (src/post/main.cpp:204-253): the case of
//            the deck, the state and time of a solution file, its L2 errors
//
// Deck keys (as in the reference, src/exec/main.cpp:52-119,
// src/solver/base.cpp:20-67, src/physics/base/base.cpp:25-32):
//   [Mesh]     file = "mesh.h5": a mesh file of the reference's format
//              (Mesh::read_mesh, src/mesh/mesh.cpp:79-204; read by
//              dg_mesh_read_h5; a relative path is taken from the working
//              directory, as the reference opens it);
//              when no such file exists and the name is the reference's
//              "...cube_<N>.h5", the periodic N^3 box on [0,1]^3 that file
//              holds is generated instead; or
//              periodic_box = [nx, ny, nz], origin = [..], length = [..]
//              2D ([Physics] dim = 2): a quadrilateral mesh file, a missing
//              "...box_<N>x<M>.h5" (the periodic N x M box on [-5, 5]^2 of the
//              reference's 2D vortex study), or periodic_box = [nx, ny]
//   [Numerics] order, basis = "LagrangeHex" (2D: "LagrangeQuad")
//   [Stepper]  type = "FE" | "RK4" (default "FE"), timestep, end;
//              extensions: cfl (derive timestep from the IC), steps (count)
//   [Physics]  name = "Euler", dim = 3 or 2, gamma = 1.4, GasConstant = 287.05,
//              convective_flux_fcn = "LaxFriedrichs" | "HLLC"
//   [InitialCondition] name, data
//   [Output]   as the reference (src/exec/main.cpp:105-112), the final state
//              is written to data.h5 in the writer's schema
//              (dg_solution_write_h5); disable_all_outputs = true skips it;
//              (extensions) solution_file = "path" (instead of data.h5);
//              print_every = N; state_file = "path" (binary checkpoint at
//              the end: int64 ne, nb, 5, double time, then Uc [ne][nb][5]);
//              restart_file = "path" (start from such a checkpoint, or from a
//              *.h5 solution file of the writer's schema, instead of the
//              initial condition; with `end` the run stops at that time, with
//              `steps` it takes that many more); json = true (one JSON line
//              of run metrics at the end)
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <regex>
#include <string>
#include <vector>

#include "../../include/dg_b200.h"
#include "toml_lite.h"

namespace {

struct Solver;

// StepperBase / FE / RK4 of src/numerics/timestepping/stepper.h:14-90; the
// step itself is the device path behind the C ABI.
struct StepperBase {
    virtual ~StepperBase() = default;
    void set_time_step(double dt_) { dt = dt_; }
    void set_final_time(double t) { tfinal = t; }
    double get_time_step() const { return dt; }
    double get_tfinal() const { return tfinal; }
    virtual int take_time_step(Solver& solver) = 0;
    double dt = 0.0, tfinal = 0.0;
};

struct Solver {
    dg_ctx* ctx = nullptr;
    dg_ctx2d* ctx2 = nullptr;  // a 2D case (Solver<2>) instead
    double time = 0.0;
    std::vector<double> restart_state;  // [ne][nb][5] from a checkpoint, else empty
    long num_iterations = 0;
    int print_every = 0;
    std::unique_ptr<StepperBase> stepper;

    // Solver::solve, src/solver/base.cpp:377-399
    int solve()
    {
        const auto t0 = std::chrono::steady_clock::now();
        for (long it = 0; it < num_iterations; ++it) {
            int rc = stepper->take_time_step(*this);
            if (rc) return rc;
            if (print_every > 0 && (it + 1) % print_every == 0) std::printf("Time = %.10g\n", time);
        }
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("Time to Solution: %.6f s (%ld steps)\n", sec, num_iterations);
        return DG_OK;
    }
};

struct RK4Gpu : StepperBase {
    int take_time_step(Solver& s) override
    {
        const int rc = s.ctx2 ? dg2d_rk4_steps(s.ctx2, dt, 1) : dg_rk4_steps(s.ctx, dt, 1);
        s.time += dt;  // stage times t, t+dt/2, t+dt/2, t+dt (stepper.cpp:98,125)
        return rc;
    }
};

struct FEGpu : StepperBase {
    int take_time_step(Solver& s) override
    {
        const int rc = s.ctx2 ? dg2d_fe_steps(s.ctx2, dt, 1) : dg_fe_steps(s.ctx, dt, 1);
        s.time += dt;
        return rc;
    }
};

int ic_code(const std::string& name)
{
    if (name == "Uniform") return DG_IC_UNIFORM;
    if (name == "IsentropicVortex") return DG_IC_VORTEX_REF;
    if (name == "Sphere") return DG_IC_SPHERE;
    if (name == "IsentropicVortexXY") return DG_IC_VORTEX_XY;
    if (name == "TaylorGreen") return DG_IC_TAYLOR_GREEN;
    throw std::runtime_error("unknown [InitialCondition] name " + name);
}

bool file_exists(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    return static_cast<bool>(f);
}

bool ends_with(const std::string& s, const std::string& tail)
{
    return s.size() >= tail.size() && s.compare(s.size() - tail.size(), tail.size(), tail) == 0;
}

int run2d(const dgh::Toml& deck, bool check_only, const char* post);

int run(const dgh::Toml& deck, bool check_only, const char* post)
{
    if (static_cast<int>(deck.num_or("Physics", "dim", 3)) == 2) return run2d(deck, check_only, post);
    // ---- mesh ----
    int n[3] = {0, 0, 0};
    double x0[3] = {0, 0, 0}, len[3] = {1, 1, 1};
    std::string mesh_file;
    if (deck.has("Mesh", "periodic_box")) {
        const auto b = deck.nums("Mesh", "periodic_box");
        if (b.size() != 3) throw std::runtime_error("[Mesh] periodic_box needs 3 entries");
        for (int i = 0; i < 3; ++i) n[i] = static_cast<int>(b[i]);
        if (deck.has("Mesh", "origin")) { auto o = deck.nums("Mesh", "origin"); for (int i = 0; i < 3; ++i) x0[i] = o.at(i); }
        if (deck.has("Mesh", "length")) { auto l = deck.nums("Mesh", "length"); for (int i = 0; i < 3; ++i) len[i] = l.at(i); }
    } else {
        const std::string file = deck.str("Mesh", "file");
        const std::string& path = file;
        std::smatch m;
        if (file_exists(path)) {
            mesh_file = path;
        } else if (std::regex_search(file, m, std::regex("cube_([0-9]+)\\.h5$"))) {
            n[0] = n[1] = n[2] = std::stoi(m[1]);
        } else {
            throw std::runtime_error("[Mesh] file " + path + " not found");
        }
    }
    // ---- numerics / physics ----
    const int order = static_cast<int>(deck.num("Numerics", "order"));
    const std::string basis = deck.str_or("Numerics", "basis", "LagrangeHex");
    if (basis != "LagrangeHex") throw std::runtime_error("[Numerics] basis " + basis + " is not on the device path");
    if (deck.str_or("Physics", "name", "Euler") != "Euler") throw std::runtime_error("[Physics] name must be Euler");
    if (static_cast<int>(deck.num_or("Physics", "dim", 3)) != 3) throw std::runtime_error("[Physics] dim must be 2 or 3");
    const double gamma = deck.num_or("Physics", "gamma", 1.4);
    const double R = deck.num_or("Physics", "GasConstant", 287.05);
    const std::string flux_name = deck.str_or("Physics", "convective_flux_fcn", "LaxFriedrichs");
    int flux = DG_FLUX_LAX_FRIEDRICHS;
    if (flux_name == "HLLC") flux = DG_FLUX_HLLC;
    else if (flux_name != "LaxFriedrichs") throw std::runtime_error("unknown convective_flux_fcn " + flux_name);
    const std::string ic_name = deck.str("InitialCondition", "name");
    const int ic = ic_code(ic_name);
    std::vector<double> ic_data = deck.has("InitialCondition", "data") ? deck.nums("InitialCondition", "data")
                                                                          : std::vector<double>();
    if (ic_data.size() > 10) throw std::runtime_error("[InitialCondition] data holds at most 10 values");
    const std::string stype = deck.str_or("Stepper", "type", "FE");
    if (stype != "FE" && stype != "RK4") throw std::runtime_error("[Stepper] type must be FE or RK4");

    int nn = 0, ne = 0, nf = 0;
    std::vector<double> coords;
    std::vector<unsigned> e2n, faces;
    if (!mesh_file.empty()) {
        int dim = 0, qorder = 0, npe = 0;
        if (dg_mesh_read_h5(mesh_file.c_str(), &dim, &qorder, &npe, &nn, nullptr, &ne, nullptr, &nf, nullptr))
            throw std::runtime_error(dg_last_error(nullptr));
        if (dim != 3 || qorder != 1 || npe != 8)
            throw std::runtime_error("[Mesh] file " + mesh_file + ": dimension " + std::to_string(dim) + ", QOrder " +
                                     std::to_string(qorder) + ", " + std::to_string(npe) +
                                     " nodes per element; the device path takes linear hexahedra (3, 1, 8)");
        coords.resize(static_cast<size_t>(nn) * 3);
        e2n.resize(static_cast<size_t>(ne) * 8);
        faces.resize(static_cast<size_t>(nf) * 8);
        if (dg_mesh_read_h5(mesh_file.c_str(), &dim, &qorder, &npe, &nn, coords.data(), &ne, e2n.data(), &nf,
                            faces.data()))
            throw std::runtime_error(dg_last_error(nullptr));
        std::printf("case: %s (%d hex elements, %d interior faces), p=%d, %s flux, %s, IC %s\n", mesh_file.c_str(), ne,
                    nf, order, flux_name.c_str(), stype.c_str(), ic_name.c_str());
    } else {
        std::printf("case: %dx%dx%d periodic hex, p=%d, %s flux, %s, IC %s\n", n[0], n[1], n[2], order,
                    flux_name.c_str(), stype.c_str(), ic_name.c_str());
    }
    if (check_only) return 0;

    if (mesh_file.empty()) {
        if (dg_mesh_periodic_box(n, x0, len, 0, &nn, nullptr, &ne, nullptr, &nf, nullptr))
            throw std::runtime_error("bad box");
        coords.resize(static_cast<size_t>(nn) * 3);
        e2n.resize(static_cast<size_t>(ne) * 8);
        faces.resize(static_cast<size_t>(nf) * 8);
        dg_mesh_periodic_box(n, x0, len, 0, &nn, coords.data(), &ne, e2n.data(), &nf, faces.data());
    }
    dg_mesh_desc md{nn, coords.data(), ne, e2n.data(), nf, faces.data(), 0};
    dg_case_desc cd{order, flux, gamma, R, DG_PREC_FP64, 0};

    Solver solver;
    if (dg_create(&cd, &md, &solver.ctx)) throw std::runtime_error(std::string("dg_create: ") + dg_last_error(nullptr));
    const int nb = dg_num_basis(solver.ctx);
    std::vector<double> Uc(static_cast<size_t>(ne) * nb * 5);
    if (post) {
        // run_post (src/post/main.cpp:204-253): the solution file's state and
        // time, then get_error
        int fne = 0, fnb = 0, fns = 0;
        double t = 0.0;
        if (dg_solution_read_h5(post, &fne, &fnb, &fns, &t, nullptr)) throw std::runtime_error(dg_last_error(nullptr));
        if (fne != ne || fnb != nb || fns != 5)
            throw std::runtime_error(std::string(post) + " does not hold a state of this mesh and order");
        if (dg_solution_read_h5(post, &fne, &fnb, &fns, &t, Uc.data())) throw std::runtime_error(dg_last_error(nullptr));
        if (dg_set_state(solver.ctx, Uc.data())) throw std::runtime_error(dg_last_error(solver.ctx));
        std::printf("time=%.17g\n", t);
        double err[5];
        if (dg_l2_error(solver.ctx, ic, ic_data.data(), static_cast<int>(ic_data.size()), t, err))
            throw std::runtime_error(std::string("l2 error: ") + dg_last_error(solver.ctx));
        for (int k = 0; k < 5; ++k) std::printf("norm_total_error(%d)=%.*e\n", k, DECIMAL_DIG, err[k]);
        dg_destroy(solver.ctx);
        return 0;
    }
    // Solver::init_state_from_fcn (L2 projection), base.cpp:113-223
    if (dg_project_ic(solver.ctx, ic, ic_data.data(), static_cast<int>(ic_data.size()), 0.0, Uc.data()))
        throw std::runtime_error(std::string("dg_project_ic: ") + dg_last_error(solver.ctx));
    const bool restart = deck.has("Output", "restart_file");
    if (restart) {
        // the time step still comes from the deck (or the CFL on the initial
        // condition), so a resumed run takes the same steps as an unbroken one
        const std::string path = deck.str("Output", "restart_file");
        std::vector<double> U0(Uc.size());
        double t = 0.0;
        if (ends_with(path, ".h5")) {
            // a solution file of the writer's schema (Solver::read_in_coefficients, base.cpp:234-279)
            int fne = 0, fnb = 0, fns = 0;
            if (dg_solution_read_h5(path.c_str(), &fne, &fnb, &fns, &t, nullptr))
                throw std::runtime_error(dg_last_error(nullptr));
            if (fne != ne || fnb != nb || fns != 5)
                throw std::runtime_error("restart_file " + path + " does not hold a state of this mesh and order");
            if (dg_solution_read_h5(path.c_str(), &fne, &fnb, &fns, &t, U0.data()))
                throw std::runtime_error(dg_last_error(nullptr));
        } else {
            std::ifstream f(path, std::ios::binary);
            long long hdr[3] = {0, 0, 0};
            f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
            f.read(reinterpret_cast<char*>(&t), sizeof(double));
            if (!f || hdr[0] != ne || hdr[1] != nb || hdr[2] != 5)
                throw std::runtime_error("restart_file " + path + " does not hold a state of this mesh and order");
            f.read(reinterpret_cast<char*>(U0.data()), static_cast<std::streamsize>(U0.size() * sizeof(double)));
            if (!f) throw std::runtime_error("restart_file " + path + " is truncated");
        }
        solver.time = t;
        solver.restart_state = std::move(U0);
    }

    double dt = deck.num_or("Stepper", "timestep", 0.0);
    if (deck.has("Stepper", "cfl")) {
        if (dg_cfl_time_step(solver.ctx, Uc.data(), deck.num("Stepper", "cfl"), &dt))
            throw std::runtime_error(std::string("cfl: ") + dg_last_error(solver.ctx));
    }
    if (!(dt > 0.0)) throw std::runtime_error("[Stepper] needs timestep > 0 (or cfl)");
    if (deck.has("Stepper", "steps")) {
        solver.num_iterations = static_cast<long>(deck.num("Stepper", "steps"));
    } else {
        // num_iterations = (int)(tfinal / dt), base.cpp:383; after a restart,
        // the steps left to that end time
        const double end = deck.num("Stepper", "end");
        solver.num_iterations = static_cast<int>(end / dt) - (restart ? static_cast<long>(solver.time / dt + 0.5) : 0);
        if (solver.num_iterations < 0) solver.num_iterations = 0;
    }
    if (restart && dg_set_state(solver.ctx, solver.restart_state.data()))
        throw std::runtime_error(std::string("dg_set_state: ") + dg_last_error(solver.ctx));
    if (stype == "RK4") solver.stepper = std::make_unique<RK4Gpu>();
    else solver.stepper = std::make_unique<FEGpu>();
    solver.stepper->set_time_step(dt);
    solver.stepper->set_final_time(dt * solver.num_iterations);
    solver.print_every = static_cast<int>(deck.num_or("Output", "print_every", 0));
    std::printf("timestep = %.17g, number of iterations = %ld, DOF = %lld\n", dt, solver.num_iterations,
                static_cast<long long>(ne) * nb * 5);

    const auto t0 = std::chrono::steady_clock::now();
    int rc = solver.solve();
    if (rc) throw std::runtime_error(std::string("solve: ") + dg_last_error(solver.ctx));
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double dof = static_cast<double>(ne) * nb * 5;
    const int stages = stype == "RK4" ? 4 : 1;
    std::string json = "{\"dof\": " + std::to_string(static_cast<long long>(dof)) +
                       ", \"order\": " + std::to_string(order) + ", \"steps\": " + std::to_string(solver.num_iterations) +
                       ", \"stages_per_step\": " + std::to_string(stages) + ", \"wall_s\": " + std::to_string(wall) +
                       ", \"dof_stage_per_s\": " + std::to_string(wall > 0 ? dof * stages * solver.num_iterations / wall : 0.0);
    char tbuf[64];
    std::snprintf(tbuf, sizeof(tbuf), "%.17g", solver.time);
    json += std::string(", \"time\": ") + tbuf;

    // post: volume-normalised L2 error against the exact solution
    // (get_error, src/post/main.cpp:30-201); TaylorGreen has none: kinetic energy instead
    if (ic == DG_IC_TAYLOR_GREEN) {
        double ke = 0.0;
        dg_kinetic_energy(solver.ctx, &ke);
        std::printf("kinetic_energy=%.*e\n", DECIMAL_DIG, ke);
        std::snprintf(tbuf, sizeof(tbuf), "%.17g", ke);
        json += std::string(", \"kinetic_energy\": ") + tbuf;
    } else {
        double err[5];
        if (dg_l2_error(solver.ctx, ic, ic_data.data(), static_cast<int>(ic_data.size()), solver.time, err))
            throw std::runtime_error(std::string("l2 error: ") + dg_last_error(solver.ctx));
        for (int s = 0; s < 5; ++s) std::printf("norm_total_error(%d)=%.*e\n", s, DECIMAL_DIG, err[s]);
        json += ", \"l2_error\": [";
        for (int s = 0; s < 5; ++s) {
            std::snprintf(tbuf, sizeof(tbuf), "%s%.17g", s ? ", " : "", err[s]);
            json += tbuf;
        }
        json += "]";
    }
    const bool outputs = !(deck.has("Output", "disable_all_outputs") && deck.boolean("Output", "disable_all_outputs"));
    if (outputs || deck.has("Output", "state_file")) dg_get_state(solver.ctx, Uc.data());
    if (outputs) {
        // Writer("data.h5", ...) after the solve, src/exec/main.cpp:105-112
        const std::string out = deck.has("Output", "solution_file") ? deck.str("Output", "solution_file") : "data.h5";
        if (dg_solution_write_h5(out.c_str(), &md, order, Uc.data(), solver.time))
            throw std::runtime_error(dg_last_error(nullptr));
        std::printf("solution written to %s\n", out.c_str());
    }
    if (deck.has("Output", "state_file")) {
        std::ofstream f(deck.str("Output", "state_file"), std::ios::binary);
        const long long hdr[3] = {ne, nb, 5};
        f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
        f.write(reinterpret_cast<const char*>(&solver.time), sizeof(double));
        f.write(reinterpret_cast<const char*>(Uc.data()), static_cast<std::streamsize>(Uc.size() * sizeof(double)));
    }
    if (deck.has("Output", "json") && deck.boolean("Output", "json")) std::printf("%s}\n", json.c_str());
    dg_destroy(solver.ctx);
    return 0;
}

// the 2D case (run_solver<2>, src/exec/main.cpp:52-119): quadrilateral
// meshes, LagrangeQuad, the dg2d_* entry points
int run2d(const dgh::Toml& deck, bool check_only, const char* post)
{
    int n[2] = {0, 0};
    double x0[2] = {-5.0, -5.0}, len[2] = {10.0, 10.0};
    std::string mesh_file;
    if (deck.has("Mesh", "periodic_box")) {
        const auto b = deck.nums("Mesh", "periodic_box");
        if (b.size() != 2) throw std::runtime_error("[Mesh] periodic_box needs 2 entries in 2D");
        for (int i = 0; i < 2; ++i) n[i] = static_cast<int>(b[i]);
        if (deck.has("Mesh", "origin")) { auto o = deck.nums("Mesh", "origin"); for (int i = 0; i < 2; ++i) x0[i] = o.at(i); }
        if (deck.has("Mesh", "length")) { auto l = deck.nums("Mesh", "length"); for (int i = 0; i < 2; ++i) len[i] = l.at(i); }
    } else {
        const std::string file = deck.str("Mesh", "file");
        std::smatch m;
        if (file_exists(file)) {
            mesh_file = file;
        } else if (std::regex_search(file, m, std::regex("box_([0-9]+)x([0-9]+)\\.h5$"))) {
            // the reference's 2D vortex boxes: periodic on [-5, 5]^2
            n[0] = std::stoi(m[1]);
            n[1] = std::stoi(m[2]);
        } else {
            throw std::runtime_error("[Mesh] file " + file + " not found");
        }
    }
    const int order = static_cast<int>(deck.num("Numerics", "order"));
    const std::string basis = deck.str_or("Numerics", "basis", "LagrangeQuad");
    if (basis != "LagrangeQuad") throw std::runtime_error("[Numerics] basis " + basis + " is not on the device path (2D: LagrangeQuad)");
    if (deck.str_or("Physics", "name", "Euler") != "Euler") throw std::runtime_error("[Physics] name must be Euler");
    const double gamma = deck.num_or("Physics", "gamma", 1.4);
    const double R = deck.num_or("Physics", "GasConstant", 287.05);
    const std::string flux_name = deck.str_or("Physics", "convective_flux_fcn", "LaxFriedrichs");
    int flux = DG_FLUX_LAX_FRIEDRICHS;
    if (flux_name == "HLLC") flux = DG_FLUX_HLLC;
    else if (flux_name != "LaxFriedrichs") throw std::runtime_error("unknown convective_flux_fcn " + flux_name);
    const std::string ic_name = deck.str("InitialCondition", "name");
    int ic = DG_IC_VORTEX_2D;
    if (ic_name == "Uniform") ic = DG_IC_UNIFORM;
    else if (ic_name == "IsentropicVortexXY") ic = DG_IC_VORTEX_XY;
    else if (ic_name != "IsentropicVortex") throw std::runtime_error("[InitialCondition] name " + ic_name + " has no 2D form");
    std::vector<double> ic_data = deck.has("InitialCondition", "data") ? deck.nums("InitialCondition", "data")
                                                                          : std::vector<double>();
    const std::string stype = deck.str_or("Stepper", "type", "FE");
    if (stype != "FE" && stype != "RK4") throw std::runtime_error("[Stepper] type must be FE or RK4");
    if (deck.has("Stepper", "cfl")) throw std::runtime_error("[Stepper] cfl: the 2D path takes timestep");

    int nn = 0, ne = 0, nf = 0;
    std::vector<double> coords;
    std::vector<unsigned> e2n, faces;
    if (!mesh_file.empty()) {
        int dim = 0, qorder = 0, npe = 0;
        if (dg_mesh_read_h5(mesh_file.c_str(), &dim, &qorder, &npe, &nn, nullptr, &ne, nullptr, &nf, nullptr))
            throw std::runtime_error(dg_last_error(nullptr));
        if (dim != 2 || qorder != 1 || npe != 4)
            throw std::runtime_error("[Mesh] file " + mesh_file + ": dimension " + std::to_string(dim) + ", QOrder " +
                                     std::to_string(qorder) + ", " + std::to_string(npe) +
                                     " nodes per element; the 2D path takes linear quadrilaterals (2, 1, 4)");
        coords.resize(static_cast<size_t>(nn) * 2);
        e2n.resize(static_cast<size_t>(ne) * 4);
        faces.resize(static_cast<size_t>(nf) * 8);
        if (dg_mesh_read_h5(mesh_file.c_str(), &dim, &qorder, &npe, &nn, coords.data(), &ne, e2n.data(), &nf,
                            faces.data()))
            throw std::runtime_error(dg_last_error(nullptr));
        std::printf("case: %s (%d quadrilaterals, %d interior faces), p=%d, %s flux, %s, IC %s\n", mesh_file.c_str(),
                    ne, nf, order, flux_name.c_str(), stype.c_str(), ic_name.c_str());
    } else {
        std::printf("case: %dx%d periodic quad, p=%d, %s flux, %s, IC %s\n", n[0], n[1], order, flux_name.c_str(),
                    stype.c_str(), ic_name.c_str());
    }
    if (check_only) return 0;
    if (mesh_file.empty()) {
        if (dg_mesh2d_periodic_box(n, x0, len, 0, &nn, nullptr, &ne, nullptr, &nf, nullptr)) throw std::runtime_error("bad box");
        coords.resize(static_cast<size_t>(nn) * 2);
        e2n.resize(static_cast<size_t>(ne) * 4);
        faces.resize(static_cast<size_t>(nf) * 8);
        dg_mesh2d_periodic_box(n, x0, len, 0, &nn, coords.data(), &ne, e2n.data(), &nf, faces.data());
    }
    dg_mesh2d_desc md{nn, coords.data(), ne, e2n.data(), nf, faces.data(), 0};
    dg_case_desc cd{order, flux, gamma, R, DG_PREC_FP64, 0};
    Solver solver;
    if (dg2d_create(&cd, &md, &solver.ctx2)) throw std::runtime_error(std::string("dg2d_create: ") + dg_last_error(nullptr));
    const int nb = dg2d_num_basis(solver.ctx2);
    std::vector<double> Uc(static_cast<size_t>(ne) * nb * 4);
    if (post) {
        int fne = 0, fnb = 0, fns = 0;
        double t = 0.0;
        if (dg_solution_read_h5(post, &fne, &fnb, &fns, &t, nullptr)) throw std::runtime_error(dg_last_error(nullptr));
        if (fne != ne || fnb != nb || fns != 4)
            throw std::runtime_error(std::string(post) + " does not hold a 2D state of this mesh and order");
        if (dg_solution_read_h5(post, &fne, &fnb, &fns, &t, Uc.data())) throw std::runtime_error(dg_last_error(nullptr));
        if (dg2d_set_state(solver.ctx2, Uc.data())) throw std::runtime_error(dg2d_last_error(solver.ctx2));
        std::printf("time=%.17g\n", t);
        double err[4];
        if (dg2d_l2_error(solver.ctx2, ic, ic_data.data(), static_cast<int>(ic_data.size()), t, err))
            throw std::runtime_error(std::string("l2 error: ") + dg2d_last_error(solver.ctx2));
        for (int k = 0; k < 4; ++k) std::printf("norm_total_error(%d)=%.*e\n", k, DECIMAL_DIG, err[k]);
        dg2d_destroy(solver.ctx2);
        return 0;
    }
    if (dg2d_project_ic(solver.ctx2, ic, ic_data.data(), static_cast<int>(ic_data.size()), 0.0, Uc.data()))
        throw std::runtime_error(std::string("dg2d_project_ic: ") + dg2d_last_error(solver.ctx2));
    const bool restart = deck.has("Output", "restart_file");
    if (restart) {
        const std::string path = deck.str("Output", "restart_file");
        int fne = 0, fnb = 0, fns = 0;
        double t = 0.0;
        if (!ends_with(path, ".h5")) throw std::runtime_error("restart_file: the 2D path resumes from *.h5 solution files");
        if (dg_solution_read_h5(path.c_str(), &fne, &fnb, &fns, &t, nullptr)) throw std::runtime_error(dg_last_error(nullptr));
        if (fne != ne || fnb != nb || fns != 4)
            throw std::runtime_error("restart_file " + path + " does not hold a state of this mesh and order");
        if (dg_solution_read_h5(path.c_str(), &fne, &fnb, &fns, &t, Uc.data())) throw std::runtime_error(dg_last_error(nullptr));
        if (dg2d_set_state(solver.ctx2, Uc.data())) throw std::runtime_error(dg2d_last_error(solver.ctx2));
        solver.time = t;
    }
    const double dt = deck.num_or("Stepper", "timestep", 0.0);
    if (!(dt > 0.0)) throw std::runtime_error("[Stepper] needs timestep > 0");
    if (deck.has("Stepper", "steps")) {
        solver.num_iterations = static_cast<long>(deck.num("Stepper", "steps"));
    } else {
        const double end = deck.num("Stepper", "end");
        solver.num_iterations = static_cast<int>(end / dt) - (restart ? static_cast<long>(solver.time / dt + 0.5) : 0);
        if (solver.num_iterations < 0) solver.num_iterations = 0;
    }
    if (stype == "RK4") solver.stepper = std::make_unique<RK4Gpu>();
    else solver.stepper = std::make_unique<FEGpu>();
    solver.stepper->set_time_step(dt);
    solver.stepper->set_final_time(dt * solver.num_iterations);
    solver.print_every = static_cast<int>(deck.num_or("Output", "print_every", 0));
    std::printf("timestep = %.17g, number of iterations = %ld, DOF = %lld\n", dt, solver.num_iterations,
                static_cast<long long>(ne) * nb * 4);
    const auto t0 = std::chrono::steady_clock::now();
    if (solver.solve()) throw std::runtime_error(std::string("solve: ") + dg2d_last_error(solver.ctx2));
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double err[4] = {0, 0, 0, 0};
    if (ic != DG_IC_UNIFORM || ic_data.size() >= 4) {
        if (dg2d_l2_error(solver.ctx2, ic, ic_data.data(), static_cast<int>(ic_data.size()), solver.time, err))
            throw std::runtime_error(std::string("l2 error: ") + dg2d_last_error(solver.ctx2));
        for (int s = 0; s < 4; ++s) std::printf("norm_total_error(%d)=%.*e\n", s, DECIMAL_DIG, err[s]);
    }
    const bool outputs = !(deck.has("Output", "disable_all_outputs") && deck.boolean("Output", "disable_all_outputs"));
    if (outputs) {
        if (dg2d_get_state(solver.ctx2, Uc.data())) throw std::runtime_error(dg2d_last_error(solver.ctx2));
        const std::string out = deck.has("Output", "solution_file") ? deck.str("Output", "solution_file") : "data.h5";
        if (dg2d_solution_write_h5(out.c_str(), &md, order, Uc.data(), solver.time))
            throw std::runtime_error(dg_last_error(nullptr));
        std::printf("solution written to %s\n", out.c_str());
    }
    if (deck.has("Output", "json") && deck.boolean("Output", "json")) {
        char buf[512];
        const int stages = stype == "RK4" ? 4 : 1;
        const double dof = static_cast<double>(ne) * nb * 4;
        std::snprintf(buf, sizeof(buf),
                      "{\"dim\": 2, \"dof\": %lld, \"order\": %d, \"steps\": %ld, \"stages_per_step\": %d, \"wall_s\": %.6f, "
                      "\"dof_stage_per_s\": %.6g, \"time\": %.17g, \"l2_error\": [%.17g, %.17g, %.17g, %.17g]}",
                      static_cast<long long>(dof), order, solver.num_iterations, stages, wall,
                      wall > 0 ? dof * stages * solver.num_iterations / wall : 0.0, solver.time, err[0], err[1], err[2],
                      err[3]);
        std::printf("%s\n", buf);
    }
    dg2d_destroy(solver.ctx2);
    return 0;
}

}  // namespace

int main(int argc, char* argv[])
{
    std::string deck_path = "input.toml", post_file;
    bool check_only = false, post = false;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "-input") && i + 1 < argc) deck_path = argv[++i];
        else if (!std::strcmp(argv[i], "-check")) check_only = true;
        else if (!std::strcmp(argv[i], "-post")) {
            post = true;
            post_file = i + 1 < argc && argv[i + 1][0] != '-' ? argv[++i] : "data.h5";
        }
    }
    try {
        return run(dgh::Toml::parse_file(deck_path), check_only, post ? post_file.c_str() : nullptr);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "dg_solve: %s\n", ex.what());
        return 2;
    }
}
