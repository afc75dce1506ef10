// A driver shaped like the reference's runNVE.cpp (lines 24-146), written
// against the C++ facade: reads a packing directory in the reference's
// format, runs NVE one step per NVELoop() call and writes the final state.
//
// usage: run_nve <packingDir/> <outDir/> <timeStep> <Tinject> <maxStep> <numParticles> <lj|wca|harmonic> <smooth|vv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "cudaring/DPM2D.hpp"
#include "cudaring/FileIO.hpp"

using cudaring::DPM2D;

int main(int argc, char** argv) {
  if (argc < 9) {
    std::cerr << "usage: run_nve inDir/ outDir/ dt T maxStep numParticles pot inter\n";
    return 2;
  }
  const std::string inDir = argv[1], outDir = argv[2], potType = argv[7], intType = argv[8];
  const double timeStep = atof(argv[3]), Tinject = atof(argv[4]);
  const long maxStep = atol(argv[5]), numParticles = atol(argv[6]);
  const long nDim = 2, numVertexPerParticle = 32;
  const double cutoff = 0.5, ea = 1e05, el = 20, eb = 10, ec = 1, LJcut = 1.5;
  try {
    DPM2D dpm(numParticles, nDim, numVertexPerParticle);
    if (potType == "lj") {
      dpm.setPotentialType(CR_POTENTIAL_LENNARD_JONES);
      dpm.setLJcutoff(LJcut);
    } else if (potType == "wca") {
      dpm.setPotentialType(CR_POTENTIAL_WCA);
    }
    if (intType == "smooth") {
      dpm.setInteractionType(CR_INTERACTION_VERTEX_SMOOTH);
      dpm.setNeighborType(0);
    }
    cudaring::ioDPMFile ioDPM(&dpm);
    ioDPM.readPackingFromDirectory(inDir, numParticles, nDim);
    dpm.setEnergyCosts(ea, el, eb, ec);
    ioDPM.readState(inDir, numParticles, dpm.getNumVertices(), nDim);
    const double sigma = dpm.getMeanParticleSize();
    const double timeUnit = sigma / std::sqrt(ec);
    dpm.setTimeStep(timeStep * timeUnit);
    dpm.initNVE(Tinject, true);
    const double size = 2 * dpm.getMeanVertexRadius();
    const double cutDistance = dpm.setDisplacementCutoff(cutoff, size);
    dpm.calcNeighbors(cutDistance);
    dpm.calcForceEnergy();
    dpm.resetUpdateCount();
    const double e0 = dpm.getEnergy();
    long step = 0;
    while (step != maxStep) {
      dpm.NVELoop();
      step += 1;
    }
    ioDPM.precision = 17;
    ioDPM.savePacking(outDir);
    std::printf("{\"steps\": %ld, \"updates\": %ld, \"energy0\": %.17g, \"energy\": %.17g}\n", step,
                dpm.getUpdateCount(), e0, dpm.getEnergy());
  } catch (const cudaring::Error& e) {
    std::cerr << "run_nve: " << e.what() << " (status " << e.code << ")\n";
    return 1;
  }
  return 0;
}
