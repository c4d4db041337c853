/*
 * ref_timed_main.cpp -- TEST INFRASTRUCTURE ONLY (oracle side).
 *
 * Entry point for the reference's own end-to-end GPU path, built from the reference's
 * unmodified sources (all of Src/ except main.cpp, and all of CUDA/ through ref_compat.h).
 * It does what Src/main.cpp:10-49 does -- FileParams, ReconData, the factory's
 * "Helicalfdkramprebingpu" reconstructor, reconstruct(), RawImageWriter -- and additionally
 * times reconstruct() (wall clock around a device synchronisation) so the plain FP32 GPU
 * path can be reported beside the product.  Its stdout banners are the reference's own;
 * the last line is a JSON record.
 *
 * `ref_timed <prm> pi` builds the reference's alternate configuration instead, the one its
 * factory has commented out (Src/ReconstructorAbstractFactory.cpp:19-22): the FDKReconstructor
 * over PiOriRebiner, PiOriPreWeighting, RampFilterGPU and PiOriBackprojectorGPU, all the
 * reference's own classes and kernels.
 */
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <string>

#include "Backprojector.h"
#include "DataStructs.h"
#include "FileParams.h"
#include "Filter.h"
#include "ImageWriter.h"
#include "PreWeighting.h"
#include "Rebiner.h"
#include "Reconstructor.h"
#include "ReconstructorAbstractFactory.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_timed <prm> [pi]\n");
    return 1;
  }
  FileParams* fp = new FileParams(std::string(argv[1]));
  ReconData* mr = new ReconData(*fp);
  ReconstrctorAbstractFactory* fac = new ReconstrctorAbstractFactory();
  const bool pi = argc >= 3 && std::string(argv[2]) == "pi";
  Reconstructor* recon =
      pi ? new FDKReconstructor(new PiOriRebiner(), new RampFilterGPU(), new PiOriBackprojectorGPU(),
                                new PiOriPreWeighting())
         : fac->createReconstructor("Helicalfdkramprebingpu");
  cudaDeviceSynchronize();
  auto t0 = std::chrono::steady_clock::now();
  recon->reconstruct(mr);
  cudaError_t err = cudaDeviceSynchronize();
  auto t1 = std::chrono::steady_clock::now();
  ImageWriter* w = new RawImageWriter();
  w->writeImage(mr);
  double s = std::chrono::duration<double>(t1 - t0).count();
  std::printf("{\"reconstruct_seconds\": %.6f, \"n_blocks\": %d, \"cuda_error\": %d, \"chain\": \"%s\"}\n",
              s, mr->ri_()->n_blocks(), (int)err, pi ? "pi_original" : "fan2par");
  delete w;
  delete recon;
  delete fac;
  delete mr;
  delete fp;
  return err == cudaSuccess ? 0 : 3;
}
