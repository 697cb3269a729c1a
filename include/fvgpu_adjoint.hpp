/*
 * fvgpu_adjoint.hpp -- C++ reverse-mode API over the adjoint entry points of
 * fvgpu.h (fv_adjoint_*).  Header only; errors throw std::runtime_error with
 * fv_last_error()'s message.
 *
 *   fvgpu::InflowAdjoint adj(mesh, physics, options);
 *   double loss = adj.forward(theta);                 // FP64_EXACT time loop
 *   std::vector<double> g = adj.gradient(theta);      // forward + reverse sweep
 *
 * theta = (inflow Mach, density bin 1 .. n_bins); see fv_adjoint_create.
 */
#ifndef FVGPU_ADJOINT_HPP
#define FVGPU_ADJOINT_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "fvgpu.h"

namespace fvgpu {

class InflowAdjoint {
public:
    InflowAdjoint(const fv_mesh* mesh, const fv_physics& physics, const fv_adjoint_options& options,
                  int device = 0)
        : n_params_(1 + options.n_bins) {
        int64_t sz[5];
        check(fv_mesh_sizes(mesh, sz));
        n_total_ = sz[2];
        check(fv_adjoint_create(mesh, &physics, device, &options, &a_));
    }
    InflowAdjoint(const InflowAdjoint&) = delete;
    InflowAdjoint& operator=(const InflowAdjoint&) = delete;
    ~InflowAdjoint() {
        if (a_) fv_adjoint_destroy(a_);
    }

    /* The loss of one forward run. */
    double forward(const std::vector<double>& theta) {
        need(theta);
        double loss = 0.0;
        check(fv_adjoint_run(a_, theta.data(), &loss, nullptr));
        return loss;
    }
    /* dloss/dtheta (reverse mode); the loss of the same run in *loss. */
    std::vector<double> gradient(const std::vector<double>& theta, double* loss = nullptr) {
        need(theta);
        std::vector<double> g((size_t)n_params_);
        double l = 0.0;
        check(fv_adjoint_run(a_, theta.data(), &l, g.data()));
        if (loss) *loss = l;
        return g;
    }
    /* State after the last forward run, reference numbering [n_total][4]. */
    std::vector<double> final_state() const {
        std::vector<double> q((size_t)n_total_ * 4);
        check(fv_adjoint_final_state(a_, q.data()));
        return q;
    }
    int n_params() const { return n_params_; }

private:
    static void check(int rc) {
        if (rc != FV_OK) throw std::runtime_error(std::string("fvgpu adjoint: ") + fv_last_error());
    }
    void need(const std::vector<double>& theta) const {
        if ((int)theta.size() != n_params_) throw std::invalid_argument("fvgpu adjoint: theta has the wrong size");
    }
    fv_adjoint* a_ = nullptr;
    int n_params_ = 0;
    int64_t n_total_ = 0;
};

}  // namespace fvgpu

#endif
