// Final profile of SCRIMP++ from its two phases.
//
// The reference keeps its PreSCRIMP profile and lowers it with every exact
// diagonal g > m/4, replacing an entry only on a strictly smaller distance
// (scrimppp/src/ScrimpppOrig.cpp:286-346).  PreSCRIMP itself excludes only
// |i - j| < m/4 (:190-193), so it also accepts neighbours exactly m/4 away,
// which no exact diagonal reaches.  Every other cell PreSCRIMP evaluates lies
// on an exact diagonal too, where the exact phase recomputes it (to rounding).
// So the final profile is the exact one, except where PreSCRIMP's neighbour is
// m/4 away and strictly closer than the exact phase's.
#pragma once

#include <cstdint>

namespace matrix_profile {

// d2/idx: the exact phase's profile (diagonals > excl), updated in place;
// pre_d2/pre_idx: PreSCRIMP's (+inf where no cell reached a window).
inline void merge_prescrimp_lag(int64_t PL, int64_t excl, const double* pre_d2,
                                const int64_t* pre_idx, double* d2, int64_t* idx) {
    for (int64_t w = 0; w < PL; ++w) {
        const int64_t lag = pre_idx[w] > w ? pre_idx[w] - w : w - pre_idx[w];
        if (lag == excl && pre_d2[w] < d2[w]) {
            d2[w] = pre_d2[w];
            idx[w] = pre_idx[w];
        }
    }
}

}  // namespace matrix_profile
