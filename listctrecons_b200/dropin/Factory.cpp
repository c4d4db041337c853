// ReconstrctorAbstractFactory::createReconstructor for the typed drop-in program
// (LISTCTRecons_b200).  The reference's own type names keep the reference's decision
// (Src/ReconstructorAbstractFactory.cpp:11-33): the FDKReconstructor over the fan->parallel
// rebinner, no pre-weighting, the Ram-Lak filter and the rebinned backprojector -- here the
// drop-in stages of Stages.cpp.  Two new names are matched first:
//   "Helicalfdkramprebinb200"  the whole-scan reconstructor of B200Reconstructor.cpp;
//   "Helicalfdkpiorigpu"       the reference's alternate configuration, commented out in its
//                              factory (Src/ReconstructorAbstractFactory.cpp:19-22): PiOriRebiner,
//                              PiOriPreWeighting, RampFilterGPU, PiOriBackprojectorGPU, here the
//                              drop-in stages.
// The reference's test `str.find("fdk")` is kept as it decides for every other name: it is true
// unless "fdk" starts the name.
#include <cstdlib>
#include <iostream>
#include <string>

#include "Backprojector.h"
#include "Filter.h"
#include "PreWeighting.h"
#include "Rebiner.h"
#include "Reconstructor.h"
#include "ReconstructorAbstractFactory.h"

Reconstructor* lct_make_b200_reconstructor();  // B200Reconstructor.cpp

Reconstructor* ReconstrctorAbstractFactory::createReconstructor(const std::string& str) {
  if (str == "Helicalfdkramprebinb200") return lct_make_b200_reconstructor();
  if (str == "Helicalfdkpiorigpu")
    return new FDKReconstructor(new PiOriRebiner(), new RampFilterGPU(), new PiOriBackprojectorGPU(),
                                new PiOriPreWeighting());
  if (str.find("fdk"))
    return new FDKReconstructor(new HelicalConeBeamFan2ParRebinerGPU(), new RampFilterGPU(),
                                new HelicalConeBeamFanRebinBackprojectorGPU(),
                                new NULLPreWeighting());
  std::cout << "Error happens when building reconstructor." << std::endl;
  std::exit(1);
  return nullptr;
}
