// rmhd2d.hpp -- header-only C++ facade over the C ABI (rmhd2d.h) with the
// method names of the reference's class
// (ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY/resistiveMHD_2D.hpp:9-52),
// so a reference driver program switches by replacing its #includes and
// link line:
//
//   class MyRun : public rmhd2d::ResistiveMHD2D {
//       using rmhd2d::ResistiveMHD2D::ResistiveMHD2D;
//       void initializeU() override { /* fill hostU() (nx*ny*8 doubles) */ }
//   };
//   MyRun run(cfg); run.initialize();
//   for (...) { run.oneStepRK2(); if (run.checkCalculationIsCrashed()) break;
//               totalTime += run.dt(); }
//
// Differences from the reference, by design: the configuration is a struct
// instead of link-time globals; initializeU fills a host array (hostU) that
// is uploaded with the boundary applied, as the reference drivers do at the
// end of their initializeU; errors throw rmhd2d::Error.
#pragma once

#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "rmhd2d.h"

namespace rmhd2d {

struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string &msg) : std::runtime_error(msg), status(st) {}
};

inline void check(int st, const rmhd2d_solver *s)
{
    if (st != RMHD2D_OK)
        throw Error(st, std::string(rmhd2d_status_string(st)) + ": " + rmhd2d_last_error(s));
}

class ResistiveMHD2D {
public:
    explicit ResistiveMHD2D(const rmhd2d_config &cfg) : cfg_(cfg), hU_((size_t)cfg.nx * cfg.ny * 8, 0.0)
    {
        check(rmhd2d_create(&cfg_, &s_), nullptr);
    }
    virtual ~ResistiveMHD2D() { rmhd2d_destroy(s_); }
    ResistiveMHD2D(const ResistiveMHD2D &) = delete;
    ResistiveMHD2D &operator=(const ResistiveMHD2D &) = delete;

    // The user's initial condition: fill hostU() (cell k = j + i*ny, 8 doubles each).
    virtual void initializeU() {}

    // initializeU() + upload + boundary (the reference drivers' pattern).
    void initialize()
    {
        initializeU();
        if (hU_.size() != (size_t)cfg_.nx * cfg_.ny * 8)
            throw Error(RMHD2D_ERR_INVALID, "hostU() must hold nx*ny*8 doubles");
        check(rmhd2d_set_state(s_, hU_.data(), 1), s_);
    }

    void oneStepRK2() { check(rmhd2d_step_rk2(s_), s_); }
    void run(int nsteps) { check(rmhd2d_run(s_, nsteps), s_); }

    double calculateDt()
    {
        double dt = 0.0;
        check(rmhd2d_calculate_dt(s_, &dt), s_);
        return dt;
    }
    double dt()
    {
        double dt = 0.0;
        check(rmhd2d_get_dt(s_, &dt), s_);
        return dt;
    }
    double totalTime()
    {
        double t = 0.0;
        check(rmhd2d_get_total_time(s_, &t), s_);
        return t;
    }
    bool checkCalculationIsCrashed()
    {
        int c = 0;
        check(rmhd2d_check_crashed(s_, &c), s_);
        return c != 0;
    }
    void save(const std::string &directoryname, const std::string &filenameWithoutStep, int step)
    {
        check(rmhd2d_save(s_, directoryname.c_str(), filenameWithoutStep.c_str(), step), s_);
    }
    void load(const std::string &path) { check(rmhd2d_load(s_, path.c_str()), s_); }
    std::vector<double> getU()
    {
        std::vector<double> u(hU_.size());
        check(rmhd2d_get_state(s_, u.data()), s_);
        return u;
    }
    // eta at the nx*ny cell centres (k = j + i*ny); an empty vector returns to the uniform cfg.eta.
    void setEtaTable(const std::vector<double> &eta)
    {
        if (!eta.empty() && eta.size() != (size_t)cfg_.nx * cfg_.ny)
            throw Error(RMHD2D_ERR_INVALID, "the eta table must hold nx*ny doubles");
        check(rmhd2d_set_eta_table(s_, eta.empty() ? nullptr : eta.data()), s_);
    }
    void applyBoundary() { check(rmhd2d_apply_boundary(s_), s_); }

    std::vector<double> &hostU() { return hU_; }
    const rmhd2d_config &config() const { return cfg_; }
    rmhd2d_solver *handle() { return s_; }

private:
    rmhd2d_config cfg_;
    rmhd2d_solver *s_ = nullptr;
    std::vector<double> hU_;
};

// The reference drivers' main loop (examples2D/plasmoid/main_plasmoid.cu:297-329):
// for step = 0 .. totalStep, every recordStep steps save the state as
// directoryname/filenameWithoutStep_step.bin and append "step,totalTime"
// (4 significant digits) to logfile, then take one step; stop at the first
// crashed state.  Returns the step at which the run stopped (totalStep + 1
// when it ran through) and leaves the elapsed time in totalTime.
inline int runLikeReference(ResistiveMHD2D &sim, int totalStep, int recordStep, const std::string &directoryname,
                            const std::string &filenameWithoutStep, std::ostream &logfile, double &totalTime,
                            bool echo = true)
{
    for (int step = 0; step < totalStep + 1; step++) {
        if (step % recordStep == 0) {
            sim.save(directoryname, filenameWithoutStep, step);
            logfile << std::to_string(step) << "," << std::setprecision(4) << totalTime << std::endl;
            if (echo)
                std::cout << std::to_string(step) << " step done : total time is " << std::setprecision(4)
                          << totalTime << std::endl;
        }
        sim.oneStepRK2();
        if (sim.checkCalculationIsCrashed()) {
            if (echo) std::cout << "Calculation stopped! : " << step << " steps" << std::endl;
            return step;
        }
        totalTime += sim.dt();
    }
    return totalStep + 1;
}

}  // namespace rmhd2d
