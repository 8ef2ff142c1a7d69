// The reference's driver (AMM.cu:7-95) written against include/amm_compat.hpp: the same flags,
// the same warm-up and repetitions, the same result file.  Built by tests/test_compat.py.
#include <cstdio>
#include <string>

#include "amm_compat.hpp"

static void run(host_memory& p, device_memory& dm, bool output) {
  if (p.kernel == "exact")
    powerMethod_by_exact(p, dm, output);
  else if (p.kernel == "previousAMM")
    powerMethod_by_previous(p, dm, output);
  else if (p.kernel == "proposedAMM")
    powerMethod_by_proposed(p, dm, output);
  else
    powerMethod_by_proposed_v2(p, dm, output);
}

int main(int argc, char** argv) {
  host_memory p;
  if (!p.parser(argc, argv)) return 1;
  try {
    device_memory dm(p);
    dm.write_data(p);
    dm.set_internal_randomness();
    dm.seed_start_vectors(1234ULL + p.seed);
    run(p, dm, false);  // warm-up
    cudaDeviceSynchronize();
    printf("Time,Eigenvalue,NormError\n");
    for (uint32_t i = 0; i < p.nreps; ++i) run(p, dm, true);
  } catch (const std::exception& e) {
    fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
