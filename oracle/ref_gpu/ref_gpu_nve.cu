// Times the reference's own CUDA build: farceri/cudaRing's DPM2D, compiled
// from its sources by oracle/build_ref_gpu.sh, running velocity-Verlet NVE on
// a packing stored in the reference's directory format (read by the
// reference's own ioDPMFile, include/FileIO.h:278-326, 468-474).
// Measurement infrastructure only: it reports the reference's GPU throughput
// beside the library's; nothing here is part of the library.
//
// The set-up follows the reference driver runNVE.cpp:58-130 without its file
// output: potential and interaction switches, packing + velocities from
// disk, energy costs, dt, initNVE(T, readState = true), the displacement
// cutoff 0.5 * (2 <r>), one neighbour build and force call, then NVELoop()
// steps timed with CUDA events.  shift is set false so that rebuilds follow
// the same rule as the library (checkDisplacement without the COM shift).
//
// usage: ref_gpu_nve DIR NUM_PARTICLES WARMUP STEPS DT EA EL EB POT INTER LJCUT [OUT]
//   POT = lj | wca | harmonic, INTER = smooth | vertex; OUT, when given,
//   receives the final positions then velocities as raw float64 (2 Nv each).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>

#include "include/DPM2D.h"
#include "include/FileIO.h"
#include "include/defs.h"

int main(int argc, char** argv) {
  if (argc != 12 && argc != 13) {
    std::fprintf(stderr, "usage: %s DIR NUM_PARTICLES WARMUP STEPS DT EA EL EB POT INTER LJCUT [OUT]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const long numParticles = std::atol(argv[2]);
  const long warmup = std::atol(argv[3]), steps = std::atol(argv[4]);
  const double dt = std::atof(argv[5]), ea = std::atof(argv[6]), el = std::atof(argv[7]), eb = std::atof(argv[8]);
  const std::string pot = argv[9], inter = argv[10];
  const double ljcut = std::atof(argv[11]);

  DPM2D dpm(numParticles, 2, 32);
  if (pot == "lj") {
    dpm.setPotentialType(simControlStruct::potentialEnum::lennardJones);
    dpm.setLJcutoff(ljcut);
  } else if (pot == "wca") {
    dpm.setPotentialType(simControlStruct::potentialEnum::wca);
  }
  if (inter == "smooth") {
    dpm.setInteractionType(simControlStruct::interactionEnum::vertexSmooth);
    dpm.setNeighborType(simControlStruct::neighborEnum::neighbor);
  }
  ioDPMFile io(&dpm);
  io.readPackingFromDirectory(dir + "/", numParticles, 2);
  dpm.setEnergyCosts(ea, el, eb, 1.0);
  io.readState(dir + "/", numParticles, dpm.getNumVertices(), 2);
  dpm.setTimeStep(dt);
  dpm.initNVE(0.0, true);
  dpm.shift = false;
  const double size = 2 * dpm.getMeanVertexRadius();
  const double cut = dpm.setDisplacementCutoff(0.5, size);
  dpm.calcNeighbors(cut);
  dpm.calcForceEnergy();
  dpm.resetUpdateCount();
  for (long s = 0; s < warmup; s++) dpm.NVELoop();
  cudaDeviceSynchronize();
  const long u0 = dpm.getUpdateCount();
  const double e0 = dpm.getEnergy();
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, 0);
  for (long s = 0; s < steps; s++) dpm.NVELoop();
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  const double e1 = dpm.getEnergy();
  const long nv = dpm.getNumVertices();
  if (argc == 13) {
    FILE* f = std::fopen(argv[12], "wb");
    if (!f) return 3;
    thrust::host_vector<double> pos = dpm.getVertexPositions(), vel = dpm.getVertexVelocities();
    std::fwrite(pos.data(), sizeof(double), pos.size(), f);
    std::fwrite(vel.data(), sizeof(double), vel.size(), f);
    std::fclose(f);
  }
  const cudaError_t err = cudaGetLastError();
  std::printf("{\"vertex_steps_per_s\": %.6e, \"ms_per_step\": %.6f, \"steps\": %ld, \"warmup\": %ld, "
              "\"vertices\": %ld, \"updates\": %ld, \"energy_start\": %.15e, \"energy_end\": %.15e, "
              "\"cuda_error\": \"%s\"}\n",
              (double)nv * steps / (ms * 1e-3), ms / steps, steps, warmup, nv, dpm.getUpdateCount() - u0, e0, e1,
              cudaGetErrorString(err));
  return err == cudaSuccess ? 0 : 1;
}
