// ngpb: command-line driver with the reference's flags and stage order
// (src/poisson_boltzmann.cpp:58-398): --prmfile / --potfile options.prm,
// --pqrfile molecule.pqr.  Mesh and surface are built on the host; markers,
// density map, assembly, solve, potential at atoms and energy run on the GPU.
#include <omp.h>

#include <cstdio>
#include <fstream>
#include <iostream>

#include "pb_class.h"

int main(int argc, char** argv) {
  pbh::poisson_boltzmann pb;
  pb.verbose = 1;
  if (pb.parse_options(argc, argv)) return 1;
  {
    std::ifstream in(pb.pqrfilename);
    if (pb.filetype != "pqr") {
      std::cerr << "only filetype = pqr is supported" << std::endl;
      return 1;
    }
    pb.read_atoms_from_pqr(in);
    pb.read_atoms_from_class();
  }
  if (pb.atoms.empty()) {
    std::cerr << "no atoms read from " << pb.pqrfilename << std::endl;
    return 1;
  }
  const double t0 = omp_get_wtime();
  try {
    pb.build_problem();
  } catch (const std::exception& e) {
    std::cerr << "mesh construction failed: " << e.what() << std::endl;
    return 1;
  }
  const double t1 = omp_get_wtime();
  std::cout << "  [Global] Total nodes     : " << pb.nodes.n_indep << '\n'
            << "  [Global] Hanging nodes   : " << pb.nodes.n_hang << '\n'
            << "  [Global] Total quadrants : " << pb.tmsh.size() << '\n';
  const int st = pb.run_gpu_path();
  const double t2 = omp_get_wtime();
  if (st != PBGPU_OK && st != PBGPU_NOT_CONVERGED) {
    std::cerr << "GPU path failed (status " << st << "): " << pb.last_error << std::endl;
    return 1;
  }
  if (st == PBGPU_NOT_CONVERGED) std::cerr << "[WARNING] linear solver did not converge" << std::endl;
  double ms[6] = {0, 0, 0, 0, 0, 0};
  pbgpu_get_stage_ms(pb.gpu, ms);
  std::printf("\n  solver: %d iterations, relative residual %.3e\n", pb.solve_stats.iterations,
              pb.solve_stats.rel_residual);
  std::printf("  timing [s]: mesh+surface %.3f, GPU path %.3f (markers %.4f density %.4f assemble %.4f solve %.4f "
              "atoms %.4f energy %.4f)\n",
              t1 - t0, t2 - t1, ms[0] / 1e3, ms[1] / 1e3, ms[2] / 1e3, ms[3] / 1e3, ms[4] / 1e3, ms[5] / 1e3);
  return 0;
}
