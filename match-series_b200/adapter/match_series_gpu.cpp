// match_series_gpu.cpp -- the reference's matchSeries program
// (qm/projects/electronMicroscopy/matchSeries.cpp:11-209) on the dyadic
// 2^l+1 configurator, with the GPU registration as one more deformation
// model:
//   deformationModel 22 : SSD + Dirichlet, the reference's own
//                          StandardRegistrationMultilevelDescent (CPU)
//   deformationModel 23 : the same registration with its level solve on the
//                          GPU (GpuSSDRegistrationMultilevelDescent)
// Usage: match_series_gpu <parameter file> [action], as the reference.
#include <matchSeries.h>

#include "gpu_registration.h"

typedef qc::QuocConfiguratorTraitMultiLin<double, qc::QC_2D, aol::GaussQuadrature<double, qc::QC_2D, 3> >
    DyadicConfType;

int main(int argc, char** argv) {
  try {
    aol::ParameterParser parser(argc > 1 ? argv[1] : "matchSeries.par");
    const int deformationModel = parser.getIntOrDefault("deformationModel", 23);
    switch (deformationModel) {
      case 22: {
        typedef qc::StandardRegistrationMultilevelDescent<DyadicConfType, qc::SSDRegistrationConfigurator<DyadicConfType> >
            RegisType;
        matchSeries<DyadicConfType, RegisType>(parser, argc, argv);
      } break;
      case 23:
        matchSeries<DyadicConfType, GpuSSDRegistrationMultilevelDescent<DyadicConfType> >(parser, argc, argv);
        break;
      default:
        throw aol::UnimplementedCodeException("Unknown deformationModel", __FILE__, __LINE__);
    }
  } catch (aol::Exception& el) {
    // the reference reports its exceptions and exits normally (matchSeries.cpp:204-206)
    el.dump();
  }
  return 0;
}
