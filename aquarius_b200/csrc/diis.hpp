// Standalone DIIS over caller tensors (src/convergence/diis.hpp:36-228), device resident.
#pragma once

#include <cstdint>
#include <vector>

#include "engine.hpp"

namespace ccsd {

class DiisRing {
public:
    DiisRing(Context& ctx, int order, int start, double damping);
    ~DiisRing();
    DiisRing(const DiisRing&) = delete;
    DiisRing& operator=(const DiisRing&) = delete;

    // DIIS::extrapolate(x, dx) for x = [x_0 .. x_{n-1}], dx likewise: store (x, dx), add
    // the new error-matrix row, solve the bordered system and overwrite x and dx with the
    // combinations.  Synchronises the context's stream; CCSD_ERR_SINGULAR when the
    // system stays singular after the eps retry.
    void extrapolate(const std::vector<int>& x, const std::vector<int>& dx, const double* weights);
    // coefficients of the last call by age (0 = the vector just stored); returns the
    // number of stored vectors
    int coefficients(double* c_by_age);

    Context& ctx;

private:
    struct Seg {
        int64_t off, len;
        double w;
    };
    void lay_out(const std::vector<int>& x, const std::vector<int>& dx, const double* weights);

    int order, start;
    double damping;
    bool laid_out = false;
    std::vector<int64_t> piece_len, piece_off;
    std::vector<Seg> segs;
    int64_t vec_len = 0;
    std::vector<double*> xs, dxs;
    const double** d_xs = nullptr;
    const double** d_dxs = nullptr;
    double *d_e = nullptr, *d_c = nullptr, *d_dots = nullptr;
    int* d_state = nullptr;
    int* h_state = nullptr;
    double* h_c = nullptr;
};

}  // namespace ccsd
