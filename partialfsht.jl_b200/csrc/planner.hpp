// Host planner of PartialFSHT.jl: minimal colatitude x longitude boxes, the counted cost model,
// the partition of a point set into boxes and the choice of leaf (src/Box.jl, src/Cost.jl).
// Nothing here sorts: every box and split site comes from the O(n) bucketed maximum gap.
#pragma once
#include <cstdint>
#include <vector>

namespace pf {

// SphereBox (src/Box.jl:23-30)
struct SphereBox {
    double lo = 0, hi = 0;            // colatitude extent
    double phistart = 0, phiext = 0;  // longitude arc from phistart, counter-clockwise
    bool touches_north = false, touches_south = false;
};

// CostConstants (src/Cost.jl:39-58): per-unit costs, defaults the measured ratios
struct CostConstants {
    double ring = 1.0, fft = 0.394, spread = 0.334, ft_conn = 5.18;
    bool calibrated = false;
};
CostConstants cost_constants();
void set_cost_constants(double ring, double fft, double spread, double ft_conn);  // calibrated

// bounding_box (src/Box.jl:42-73): exact colatitude min/max (clamped to [0, pi]) and the
// complement of the largest circular longitude gap
SphereBox bounding_box(const double* theta, const double* phi, int64_t n);

// cost_direct / cost_stretch (src/Cost.jl:107-142); cost_stretch is +inf for a geometry the
// stretched construction refuses at this lmax and tol
double cost_direct(int64_t npts, int lmax, int ntrans);
double cost_stretch(const SphereBox& box, int64_t npts, int lmax, int ntrans, double tol);

// partition_boxes_costed (src/Box.jl:156-200): split at the largest gap while counted cost
// falls; groups are ascending 0-based point indices
struct Partition {
    std::vector<std::vector<int32_t>> groups;
    std::vector<SphereBox> boxes;
    std::vector<double> costs;
};
void partition_boxes_costed(const double* theta, const double* phi, int64_t n, int lmax,
                            int ntrans, double tol, int maxboxes, Partition& out);

// select_method (src/Cost.jl:171-201) for AutoAlgorithm: 1 stretch, 2 direct, 3 multi-box (the
// pfsht_method values); `part` receives the partition when it was computed (maxboxes 8)
int select_method(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                  double tol, Partition* part);

}  // namespace pf
