// Host-side helpers shared by the C ABI translation units.
#pragma once
#include <cstdint>
#include <vector>

namespace lt {

// Records `msg` as this thread's last error and returns `code`.
int set_error(int code, const char* msg);

// Seeded Haar-random SU(3) links in the reference layout.
void haar_links(const int ext[4], uint64_t seed, double* out);

// MetaBiasPotential (actions/bias_potential/metadynamics.hpp:29-507): a grid of bins+1
// points over [cv_min, cv_max], well-tempered Gaussian deposits, linear interpolation and a
// quadratic wall outside the range.  mode 1 replaces the Gaussian deposit by the binned one
// (update_binned).
struct Bias
{
    double cv_min, cv_max;
    int bins;
    double bin_width, bin_width_inv, weight, width, wt, thr;
    std::vector<double> grid;
    double cv_current = 0.0;
    uint64_t exceeded = 0;
    int mode = 0;   // LT_BIAS_GAUSSIAN or LT_BIAS_BINNED

    Bias(double cv_min, double cv_max, int bins, double weight, double width, double wt, double thr);
    void update(double cv);           // the deposit of the current mode
    void update_gaussian(double cv);
    void update_binned(double cv);
    double potential(double cv) const;
    double derivative(double cv) const;
};

} // namespace lt
