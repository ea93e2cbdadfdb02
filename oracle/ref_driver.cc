// ref_driver.cc -- CPU oracle driver over the reference IBPM library.
//
// TEST INFRASTRUCTURE ONLY.  Makes the same object-construction and advance
// calls as the reference CLI (src/ibpm.cc:146-342): Grid, Geometry::load,
// BaseFlow(grid, 1, alpha), NavierStokesModel, NonlinearIBSolver(..., tol),
// geom.moveBodies, model->init, solver->init, updateOperators, refreshState,
// then `advance` per step and State::computeNetForce (src/State.cc:53-63).
// Differences from the CLI: forces are written at full precision (%.17g),
// the CG tolerance is an argument (src/IBSolver.h:79-86), no Cholesky file is
// read or written, and the steady-state step time is reported as one JSON line.
//
// usage: ref_driver -nx N -ny N -ngrid L -length X -xoffset X -yoffset X
//                   -geom FILE -Re R -dt DT -scheme rk3|euler|ab2|rk3b
//                   -nsteps K [-tol T] [-alpha DEG] [-ic restart.bin]
//                   [-out PREFIX] [-dump_every K] [-warmup W] [-cholesky_cache BASENAME]
//                   [-model nonlinear|linear|adjoint|linearperiodic|sfd] [-baseflow FILE]
//                   [-pbase PREFIX -period P] [-chi X -Delta X] [-ubf 1] [-tecplot PREFIX]
// -model selects the solver class as the CLI does (src/ibpm.cc:184-229): the
// linear models get a NavierStokesModel without base flow and the base state(s)
// from restart files (FILE, or PREFIX_<k>.bin for k < P); sfd reads its filtered
// state like the CLI (loadFilteredState of the initial condition's name).
// -ubf 1 hands the single body's motion to the base flow as the CLI's -ubf
// does (src/ibpm.cc:166-178, :300-303).  -tecplot PREFIX writes the final
// state as the CLI's Tecplot output of every level, PREFIX<step>_g<lev>.plt.
#include "ibpm.h"
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <iostream>

using namespace ibpm;

static double now_s() {
    return std::chrono::duration<double>(
        std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char* argv[]) {
    int nx = 200, ny = 200, ngrid = 1, nsteps = 10, dumpEvery = 0, warmup = 0;
    double length = 4, xoff = -2, yoff = -2, Re = 100, dt = 0.01, tol = 1e-7, alphaDeg = 0;
    std::string geomFile, scheme = "rk3", ic, out, cache, modelName = "nonlinear", baseFile, pbase, tec;
    int period = 1, ubf = 0;
    double chi = 0.02, Delta = 15.;
    for (int a = 1; a + 1 < argc; a += 2) {
        std::string k = argv[a];
        const char* v = argv[a + 1];
        if (k == "-nx") nx = atoi(v);
        else if (k == "-ny") ny = atoi(v);
        else if (k == "-ngrid") ngrid = atoi(v);
        else if (k == "-length") length = atof(v);
        else if (k == "-xoffset") xoff = atof(v);
        else if (k == "-yoffset") yoff = atof(v);
        else if (k == "-geom") geomFile = v;
        else if (k == "-Re") Re = atof(v);
        else if (k == "-dt") dt = atof(v);
        else if (k == "-scheme") scheme = v;
        else if (k == "-nsteps") nsteps = atoi(v);
        else if (k == "-tol") tol = atof(v);
        else if (k == "-alpha") alphaDeg = atof(v);
        else if (k == "-ic") ic = v;
        else if (k == "-out") out = v;
        else if (k == "-dump_every") dumpEvery = atoi(v);
        else if (k == "-warmup") warmup = atoi(v);
        else if (k == "-cholesky_cache") cache = v;
        else if (k == "-model") modelName = v;
        else if (k == "-baseflow") baseFile = v;
        else if (k == "-pbase") pbase = v;
        else if (k == "-period") period = atoi(v);
        else if (k == "-chi") chi = atof(v);
        else if (k == "-Delta") Delta = atof(v);
        else if (k == "-ubf") ubf = atoi(v);
        else if (k == "-tecplot") tec = v;
        else { std::cerr << "unknown flag " << k << std::endl; return 2; }
    }
    Scheme::SchemeType st = Scheme::RK3;
    if (scheme == "euler") st = Scheme::EULER;
    else if (scheme == "ab2") st = Scheme::AB2;
    else if (scheme == "rk3b") st = Scheme::RK3b;

    Grid grid(nx, ny, ngrid, length, xoff, yoff);
    Geometry geom;
    if (!geom.load(geomFile)) { std::cerr << "geometry load failed\n"; return 3; }
    double pi = 4. * atan(1.);
    double alpha = alphaDeg * pi / 180.;
    BaseFlow q_potential(grid, 1.0, alpha);
    if (ubf && !geom.isStationary() && geom.getNumBodies() == 1) {
        Motion* m = geom.transferMotion();
        double xC = 0, yC = 0;
        geom.transferCenter(xC, yC);
        q_potential.setMotion(*m);
        q_potential.setCenter(xC, yC);
    }
    if (ubf && geom.getNumBodies() != 1) { std::cerr << "-ubf needs exactly one body\n"; return 2; }
    const bool linear = modelName == "linear" || modelName == "linearperiodic" || modelName == "adjoint";
    NavierStokesModel* mp = linear ? new NavierStokesModel(grid, geom, Re) : new NavierStokesModel(grid, geom, Re, q_potential);
    NavierStokesModel& model = *mp;
    IBSolver* sp = NULL;
    SFDSolver* sfd = NULL;
    if (modelName == "nonlinear") {
        sp = new NonlinearIBSolver(grid, model, dt, st, tol);
    } else if (modelName == "linear") {
        State x00(grid, geom.getNumPoints());
        if (!x00.load(baseFile)) { std::cerr << "baseflow load failed\n"; return 5; }
        sp = new LinearizedIBSolver(grid, model, dt, st, tol, x00);
    } else if (modelName == "adjoint") {
        State x00(grid, geom.getNumPoints());
        if (!x00.load(baseFile)) { std::cerr << "baseflow load failed\n"; return 5; }
        sp = new AdjointIBSolver(grid, model, dt, st, tol, x00);
    } else if (modelName == "linearperiodic") {
        std::vector<State> x0;
        for (int k = 0; k < period; ++k) {
            State xk(grid, geom.getNumPoints());
            if (!xk.load(pbase + "_" + std::to_string(k) + ".bin")) { std::cerr << "periodic base load failed\n"; return 5; }
            x0.push_back(xk);
        }
        sp = new LinearizedPeriodicIBSolver(grid, model, dt, st, tol, x0, period);
    } else if (modelName == "sfd") {
        sfd = new SFDSolver(grid, model, dt, st, Delta, chi);
        sp = sfd;
    } else {
        std::cerr << "unknown model " << modelName << std::endl;
        return 2;
    }
    IBSolver& solver = *sp;

    State x(grid, geom.getNumPoints());
    x.omega = 0.; x.f = 0.; x.q = 0.;
    if (!ic.empty()) {
        if (!x.load(ic)) { std::cerr << "ic load failed\n"; return 4; }
    }
    if (sfd) sfd->loadFilteredState(ic);
    geom.moveBodies(x.time);
    model.init();
    double t0 = now_s();
    // like src/ibpm.cc:291-297: reuse <cache>_0k.cholesky when it matches, else build and save
    if (cache.empty() || !solver.load(cache)) {
        solver.init();
        if (!cache.empty()) solver.save(cache);
    }
    double tInit = now_s() - t0;
    if (!q_potential.isStationary()) q_potential.setAlphaMag(x.time);
    model.updateOperators(x.time);
    model.refreshState(x);

    FILE* ff = NULL;
    if (!out.empty()) ff = fopen((out + ".forces").c_str(), "w");
    double tSteps = 0;
    int timed = 0;
    for (int i = 1; i <= nsteps; ++i) {
        double s0 = now_s();
        solver.advance(x);
        double s1 = now_s();
        if (i > warmup) { tSteps += s1 - s0; ++timed; }
        double xF, yF;
        x.computeNetForce(xF, yF);
        double drag = xF * cos(alpha) + yF * sin(alpha);
        double lift = -xF * sin(alpha) + yF * cos(alpha);
        if (ff) fprintf(ff, "%d %.17g %.17g %.17g %.17g %.17g\n", x.timestep, x.time, xF, yF, 2 * drag, 2 * lift);
        if (dumpEvery > 0 && !out.empty() && (i % dumpEvery == 0)) {
            char buf[64];
            snprintf(buf, sizeof(buf), "_%05d.bin", x.timestep);
            x.save(out + buf);
        }
    }
    if (ff) fclose(ff);
    if (!out.empty()) x.save(out + "_final.bin");
    if (!tec.empty()) {
        // the CLI's Tecplot output with -tecplotallgrids (src/ibpm.cc:310-311) of the final state
        OutputTecplot tecplot(tec + "%05d.plt", "Test run, step%05d", true);
        tecplot.setFilename(tec + "%05d_g%01d.plt");
        tecplot.doOutput(x);
    }
    printf("{\"init_s\": %.6f, \"timed_steps\": %d, \"step_s\": %.6f, \"steps_per_s\": %.6f}\n",
           tInit, timed, tSteps, timed > 0 ? timed / tSteps : 0.0);
    return 0;
}
