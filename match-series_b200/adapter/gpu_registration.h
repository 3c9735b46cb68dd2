// gpu_registration.h -- the drop-in: a RegistrationType for the reference's
// series matching whose level solve runs on the B200 through libmsgpu.
//
// The reference plugs registrations into SeriesMatching / matchSeries<>()
// (qm/projects/electronMicroscopy/matchSeries.h:17-800, 1249-1320) through
// the template concept RegistrationType, and its multilevel descent calls the
// virtual descentOnCurrentGrid() once per level (qm/modules/quoc/
// quocDescent.h:79-81, registration.h:1092-1112).  This class is the
// reference's StandardRegistrationMultilevelDescent with the SSD data term
// and the Dirichlet regulariser on the dyadic 2^l+1 configurator, with that
// one member replaced: the level's gradient flow (findTransformation,
// registration.h:967-1021) is msgpu_gd_level.  Everything else -- parameter
// file, image loading and preparation, prolongation between levels,
// composition, averaging, the files written -- is the reference's own code.
// With msgpu's default sum order the GPU solve is the reference's solve bit
// for bit, so the files this writes are the ones the reference writes.
// Errors come back as aol::Exception with libmsgpu's message, as the
// reference reports its own failures.
#ifndef MSGPU_GPU_REGISTRATION_H
#define MSGPU_GPU_REGISTRATION_H

#include <registration.h>

#include <fstream>
#include <vector>

#include "msgpu.h"

template <typename ConfiguratorType>
class GpuSSDRegistrationMultilevelDescent
    : public qc::StandardRegistrationMultilevelDescent<ConfiguratorType,
                                                       qc::SSDRegistrationConfigurator<ConfiguratorType> > {
  typedef qc::StandardRegistrationMultilevelDescent<ConfiguratorType, qc::SSDRegistrationConfigurator<ConfiguratorType> >
      Base;

 public:
  typedef typename ConfiguratorType::RealType RealType;

 private:
  msgpu_context* _ctx;

  void check(int rc, const char* file, int line) const {
    if (rc != MSGPU_OK) throw aol::Exception(_ctx ? msgpu_last_error(_ctx) : "msgpu_create failed", file, line);
  }

 public:
  explicit GpuSSDRegistrationMultilevelDescent(const aol::ParameterParser& Parser) : Base(Parser), _ctx(NULL) {
    if (Parser.hasVariable("minimizationAlgo") && Parser.getString("minimizationAlgo") != "GradientDescent")
      throw aol::Exception("the GPU level solve provides minimizationAlgo GradientDescent only", __FILE__, __LINE__);
    check(msgpu_create(Parser.getIntOrDefault("cudaDevice", 0), &_ctx), __FILE__, __LINE__);
  }

  virtual ~GpuSSDRegistrationMultilevelDescent() {
    if (_ctx) msgpu_destroy(_ctx);
  }

  // StandardRegistrationMultilevelDescent::descentOnCurrentGrid with the
  // gradient flow on the GPU (registration.h:1092-1112).
  void descentOnCurrentGrid() {
    qc::MultiArray<RealType, ConfiguratorType::Dim> phi(this->_transformation, aol::FLAT_COPY);
    const qc::SSDRegistrationConfigurator<ConfiguratorType> regisConfig(*this);
    const RealType lambda = this->getRegularizationWeight(this->_curLevel);
    this->logLevelStart(lambda);
    if (this->_disableSaving == false) regisConfig.writeInitialRegistration(*this, phi);
    // StandardRegistration's settings (registration.h:948-966, 1059-1066)
    const aol::ParameterParser& P = this->getParserReference();
    const int maxIter = P.hasVariable("maxGDIterations") ? P.getInt("maxGDIterations") : 1000;
    const double stopEps = P.hasVariable("stopEpsilon") ? P.getDouble("stopEpsilon") : 0.;
    double energy = 0.;
    int steps = 0;
    std::vector<double> log(3 * (size_t)(maxIter + 1));
    check(msgpu_gd_level_log(_ctx, this->_curLevel, this->_org_reference[this->_curLevel].getData(),
                             this->_org_template[this->_curLevel].getData(), phi[0].getData(), phi[1].getData(),
                             lambda, maxIter, stopEps, /* use_fp64 */ 1, &energy, &steps, &log[0], maxIter + 1),
          __FILE__, __LINE__);
    this->_energyOfLastSolution = energy;
    if (this->_disableSaving == false) {
      // the per-level energy log the reference's gradient descent writes
      // (gradientDescent.h:254-272): iteration - 1, lambda * E_reg, energy
      std::ofstream out(aol::strprintf("%senergy_%02d.txt", this->getSaveDirectory(), this->_curLevel).c_str());
      for (int i = 0; i <= steps && i <= maxIter; ++i)
        out << static_cast<int>(log[3 * i]) << " " << log[3 * i + 1] << " " << log[3 * i + 2] << std::endl;
      regisConfig.writeCurrentRegistration(*this, phi);
    }
  }
};

#endif  // MSGPU_GPU_REGISTRATION_H
