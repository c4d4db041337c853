// ReconstrctorAbstractFactory::createReconstructor for the typed drop-in program
// (LISTCTRecons_b200).  The reference's own type names keep the reference's decision
// (Src/ReconstructorAbstractFactory.cpp:11-33): the FDKReconstructor over the fan->parallel
// rebinner, no pre-weighting, the Ram-Lak filter and the rebinned backprojector -- here the
// drop-in stages of Stages.cpp.  One new name, "Helicalfdkramprebinb200", builds the whole-scan
// reconstructor of B200Reconstructor.cpp.  The reference's test `str.find("fdk")` is kept as it
// decides: it is true unless "fdk" starts the name, so the new name is matched first.
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
  if (str.find("fdk"))
    return new FDKReconstructor(new HelicalConeBeamFan2ParRebinerGPU(), new RampFilterGPU(),
                                new HelicalConeBeamFanRebinBackprojectorGPU(),
                                new NULLPreWeighting());
  std::cout << "Error happens when building reconstructor." << std::endl;
  std::exit(1);
  return nullptr;
}
