// Host side of the ContactSystem (reference src/collision/contact-assembly.ts):
// device buffers of the frozen active set, broadphase and CCD, and the calls
// the Newton step makes into them.
#pragma once
#include <stdexcept>

#include "../../include/closim_cuda.h"

namespace cs {

class Solver;

struct CapacityError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class ContactHost {
 public:
  double rejections = 0;
  void begin_step_and_bisect(Solver& s);
  void update_active_set(Solver& s, double* x);
  void merit_energy(Solver& s, const double* x);
  void gradient_terms(Solver& s);
  bool check_trial(Solver& s, const double* xt);
  void commit(Solver& s, const double* x);
  void kill_approach_velocity(Solver& s);
  void fill_stats(Solver& s, cs_step_stats& st);
};

void set_contact(Solver& s, const cs_contact_params* p, int floor_on, double floor_y, const float* sp, int ns,
                 const uint32_t* si, int ms);

}  // namespace cs
