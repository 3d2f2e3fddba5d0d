// ContactSystem on the device (reference src/collision/contact-assembly.ts).
#include "contact.cuh"
#include "contact_host.hpp"

namespace cs {

void set_contact(Solver&, const cs_contact_params* p, int, double, const float*, int, const uint32_t*, int) {
  if (p) throw std::invalid_argument("contact is not available in this build");
}
void ContactHost::begin_step_and_bisect(Solver&) {}
void ContactHost::update_active_set(Solver&, double*) {}
void ContactHost::merit_energy(Solver&, const double*) {}
void ContactHost::gradient_terms(Solver&) {}
bool ContactHost::check_trial(Solver&, const double*) { return true; }
void ContactHost::commit(Solver&, const double*) {}
void ContactHost::kill_approach_velocity(Solver&) {}
void ContactHost::fill_stats(Solver&, cs_step_stats&) {}

}  // namespace cs
