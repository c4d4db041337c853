// LISTCTRecons_b200 <prm> [reconstructor type]: the reference's program flow (Src/main.cpp:10-49:
// FileParams, ReconData, the factory, reconstruct, RawImageWriter) with the reconstructor type
// named on the command line instead of the fixed "Helicalfdkramprebingpu" -- so both the
// reference's name (the drop-in stages) and "Helicalfdkramprebinb200" (the whole-scan path) run
// through the reference's own interfaces.  The time of reconstruct() (wall clock, device
// synchronised) is printed as the last line, as JSON.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <iostream>
#include <string>

#include "DataStructs.h"
#include "FileParams.h"
#include "ImageWriter.h"
#include "Reconstructor.h"
#include "ReconstructorAbstractFactory.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cout << "Usage LISTCTRecons_b200 <PRM filename> [reconstructor type]" << std::endl;
    return 1;
  }
  const std::string type = argc >= 3 ? argv[2] : "Helicalfdkramprebinb200";
  FileParams* fp = new FileParams(std::string(argv[1]));
  ReconData* mr = new ReconData(*fp);
  ReconstrctorAbstractFactory* fac = new ReconstrctorAbstractFactory();
  Reconstructor* recon = fac->createReconstructor(type);
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  recon->reconstruct(mr);
  const cudaError_t err = cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  ImageWriter* w = new RawImageWriter();
  w->writeImage(mr);
  std::printf("{\"type\": \"%s\", \"reconstruct_seconds\": %.6f, \"n_blocks\": %d, \"cuda_error\": %d}\n",
              type.c_str(), std::chrono::duration<double>(t1 - t0).count(), mr->ri_()->n_blocks(),
              (int)err);
  delete w;
  delete recon;
  delete fac;
  delete mr;
  delete fp;
  return err == cudaSuccess ? 0 : 3;
}
