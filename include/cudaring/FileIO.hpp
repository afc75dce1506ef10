// cudaring/FileIO.hpp -- the reference's packing directory format for the
// C++ facade (include/FileIO.h of farceri/cudaRing, class ioDPMFile).
//
// A deformable packing is one text file per array in a directory (names and
// row layout as the reference's readers and writers use them):
//   numVertexInParticleList.dat  vertices per ring, one integer per line
//   positions.dat / velocities.dat  "x<TAB>y<TAB>" per vertex
//   radii.dat, restLengths.dat, restAngles.dat  one value per vertex
//   restAreas.dat  one value per ring;  boxSize.dat  Lx and Ly on two lines
//   shapes.dat  "area<TAB>perimeter<TAB>shape<TAB>" per ring;  params.dat
// Values are written with setprecision(14) (the reference's defs.h), read as
// the first token(s) of each line.  Only the periodic deformable form is
// handled; other shape types throw CR_ENOTSUP.
#pragma once
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "DPM2D.hpp"

namespace cudaring {

class ioDPMFile {
 public:
  explicit ioDPMFile(DPM2D* dpm) : dpm_(dpm) {}
  int precision = 14;  // digits written (defs.h: setprecision(14)); 17 round-trips doubles

  // ioDPMFile::readDeformablePackingFromDirectory (FileIO.h:278-326): ring
  // sizes, then positions, radii, rest areas / lengths / angles and the box
  void readPackingFromDirectory(const std::string& dirName, long numParticles_, long nDim_) {
    if (nDim_ != 2) throw Error("readPackingFromDirectory: only nDim == 2 is supported", CR_ENOTSUP);
    std::vector<double> nv_ = read1D(dirName + "numVertexInParticleList.dat", numParticles_);
    std::vector<long> list(nv_.size());
    long numVertices_ = 0;
    for (size_t q = 0; q < nv_.size(); q++) numVertices_ += (list[q] = (long)nv_[q]);
    dpm_->setNumVertexInParticleList(list);
    dpm_->setNumVertices(numVertices_);
    dpm_->initParticleIdList();
    dpm_->initShapeVariables(numVertices_, numParticles_);
    dpm_->initDynamicalVariables(numVertices_);
    dpm_->initNeighbors(numVertices_);
    dpm_->setVertexPositions(read2D(dirName + "positions.dat", numVertices_));
    dpm_->setVertexRadii(read1D(dirName + "radii.dat", numVertices_));
    dpm_->setRestAreas(read1D(dirName + "restAreas.dat", numParticles_));
    dpm_->setRestLengths(read1D(dirName + "restLengths.dat", numVertices_));
    dpm_->setRestAngles(read1D(dirName + "restAngles.dat", numVertices_));
    dpm_->setLengthScale();
    dpm_->setBoxSize(read1D(dirName + "boxSize.dat", 2));
    dpm_->calcParticleShape();
  }

  // ioDPMFile::readDeformableState (FileIO.h:468-474): vertex velocities
  void readState(const std::string& dirName, long numParticles_, long numVertices_, long nDim_) {
    (void)numParticles_;
    if (nDim_ != 2) throw Error("readState: only nDim == 2 is supported", CR_ENOTSUP);
    dpm_->setVertexVelocities(read2D(dirName + "velocities.dat", numVertices_));
  }

  // ioDPMFile::saveDeformablePacking + the box (FileIO.h:383-435)
  void savePacking(const std::string& dirName) {
    std::ofstream params(dirName + "params.dat");
    if (!params) throw Error("savePacking: cannot write " + dirName + "params.dat", CR_EINVAL);
    params << std::setprecision(precision);
    params << "numParticles" << "\t" << dpm_->getNumParticles() << "\n";
    params << "phi" << "\t" << dpm_->getPhi() << "\n";
    params << "phi0" << "\t" << dpm_->getPreferredPhi() << "\n";
    params << "epot" << "\t" << dpm_->getPotentialEnergy() / dpm_->getNumParticles() << "\n";
    params << "temperature" << "\t" << dpm_->getTemperature() << "\n";
    std::vector<long> list = dpm_->getNumVertexInParticleList();
    std::ofstream f(dirName + "numVertexInParticleList.dat");
    for (long n : list) f << n << "\n";
    save1D(dirName + "radii.dat", dpm_->getVertexRadii());
    save2D(dirName + "positions.dat", dpm_->getVertexPositions(), 2);
    save1D(dirName + "restAreas.dat", dpm_->getRestAreas());
    save1D(dirName + "restLengths.dat", dpm_->getRestLengths());
    save1D(dirName + "restAngles.dat", dpm_->getRestAngles());
    save2D(dirName + "velocities.dat", dpm_->getVertexVelocities(), 2);
    save2D(dirName + "shapes.dat", dpm_->getParticleShapes(), 3);
    save1D(dirName + "boxSize.dat", dpm_->getBoxSize());
  }

  // ioDPMFile::saveDeformableState (FileIO.h:504-509)
  void saveState(const std::string& dirName) {
    save2D(dirName + "positions.dat", dpm_->getVertexPositions(), 2);
    save2D(dirName + "velocities.dat", dpm_->getVertexVelocities(), 2);
    save2D(dirName + "shapes.dat", dpm_->getParticleShapes(), 3);
    save2D(dirName + "particlePos.dat", dpm_->getParticlePositions(), 2);
  }

 private:
  DPM2D* dpm_;

  static std::vector<double> read1D(const std::string& path, long rows) {
    std::ifstream f(path);
    if (!f) throw Error("cannot read " + path, CR_EINVAL);
    std::vector<double> out;
    out.reserve((size_t)rows);
    std::string line;
    while ((long)out.size() < rows && std::getline(f, line)) {
      std::istringstream s(line);
      double x;
      if (s >> x) out.push_back(x);
    }
    if ((long)out.size() != rows) throw Error(path + ": too few rows", CR_EINVAL);
    return out;
  }
  static std::vector<double> read2D(const std::string& path, long rows) {
    std::ifstream f(path);
    if (!f) throw Error("cannot read " + path, CR_EINVAL);
    std::vector<double> out;
    out.reserve((size_t)(2 * rows));
    std::string line;
    while ((long)out.size() < 2 * rows && std::getline(f, line)) {
      std::istringstream s(line);
      double x, y;
      if (s >> x >> y) {
        out.push_back(x);
        out.push_back(y);
      }
    }
    if ((long)out.size() != 2 * rows) throw Error(path + ": too few rows", CR_EINVAL);
    return out;
  }
  void save1D(const std::string& path, const std::vector<double>& v) const {
    std::ofstream f(path);
    if (!f) throw Error("cannot write " + path, CR_EINVAL);
    f << std::setprecision(precision);
    for (double x : v) f << x << "\n";
  }
  void save2D(const std::string& path, const std::vector<double>& v, int cols) const {
    std::ofstream f(path);
    if (!f) throw Error("cannot write " + path, CR_EINVAL);
    f << std::setprecision(precision);
    for (size_t r = 0; r + cols <= v.size(); r += cols) {
      for (int c = 0; c < cols; c++) f << v[r + c] << "\t";
      f << "\n";
    }
  }
};

}  // namespace cudaring
