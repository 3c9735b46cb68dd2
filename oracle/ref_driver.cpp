// ref_driver.cpp -- command-line driver over the reference's OWN templates.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile.ref against the
// quocmesh sources (their headers and .cpp files, left where they are) into
// oracle/_ref/ms_ref.  It pins the CPU restatement (oracle/ms_oracle.c) and is
// the CPU baseline that the benchmark times.  No reference source is copied:
// every operator below is instantiated from the reference headers.
//
// Arrays are raw little-endian float64 files, x fastest (quoc ILex order).
// The configurator is the dyadic 2^l+1 grid with Q1 elements and 2x2 Gauss
// quadrature (QuocConfiguratorTraitMultiLin, configurators.h:218-330), with the
// SSD data term (registration.h:1257-1273) or, for the commands ending in
// _ncc, the normalized cross-correlation data term (NCCRegistrationConfigurator,
// registration.h:1766-1780, 1909-2018), the Dirichlet regulariser
// (registration.h:677-710) and the H1 gradient flow with automatic filter
// width (gradientDescent.h:632-709).
#include <registration.h>
#include <hyperelastic.h>
#include <quocOps.h>
#include <gradientDescent.h>
#include <kernel2d.h>
#include <CSRMatrix.h>
#include <configurators.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sys/time.h>
#include <vector>

typedef double RealType;
typedef qc::QuocConfiguratorTraitMultiLin<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > ConfType;
typedef qc::ScalarArray<RealType, qc::QC_2D> ArrayType;
typedef qc::StandardRegistrationMultilevelDescent<ConfType, qc::SSDRegistrationConfigurator<ConfType> > RegisType;
typedef qc::StandardRegistrationMultilevelDescent<ConfType, qc::NCCRegistrationConfigurator<ConfType> > RegisTypeNCC;
typedef aol::H1GradientDescent<ConfType, aol::MultiVector<RealType>, qc::LinearSmoothOp<RealType> > H1Type;
typedef aol::GradientDescentWithAutomaticFilterWidth<ConfType, aol::MultiVector<RealType>, H1Type> GDType;

static int lvlN ( int l ) { return ( 1 << l ) + 1; }

static void readBin ( const char *path, RealType *dst, size_t count ) {
  FILE *f = fopen ( path, "rb" );
  if ( !f ) { fprintf ( stderr, "cannot open %s\n", path ); exit ( 2 ); }
  if ( fread ( dst, sizeof ( RealType ), count, f ) != count ) { fprintf ( stderr, "short read %s\n", path ); exit ( 2 ); }
  fclose ( f );
}

static void writeBin ( const char *path, const RealType *src, size_t count ) {
  FILE *f = fopen ( path, "wb" );
  if ( !f ) { fprintf ( stderr, "cannot write %s\n", path ); exit ( 2 ); }
  fwrite ( src, sizeof ( RealType ), count, f );
  fclose ( f );
}

static double wallSeconds ( ) {
  struct timeval tv;
  gettimeofday ( &tv, NULL );
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

// A GD solver that records, per step, the accepted tau, the filter width used
// and the energy after the step.  Only observation hooks are overridden; the
// descent itself is the reference's applySingle.
class TracingGD : public GDType {
public:
  mutable std::vector<double> energies, taus, sigmas;
  mutable std::vector<int> evals;
  mutable int evalCount;
  mutable double lastTau, lastSigma;
  TracingGD ( const qc::GridDefinition &Grid, const aol::Op<aol::MultiVector<double>, aol::Scalar<double> > &E,
              const aol::Op<aol::MultiVector<double> > &DE, int MaxIter, double StopEps )
    : GDType ( Grid, E, DE, MaxIter, 1., StopEps ), evalCount ( 0 ), lastTau ( 0 ), lastSigma ( 0 ) {}
  void writeEnergy ( const double CurrentEnergy ) const {
    if ( this->_iterations == 0 ) { energies.push_back ( CurrentEnergy ); taus.push_back ( 0 ); sigmas.push_back ( 0 ); evals.push_back ( 0 ); return; }
    energies.push_back ( CurrentEnergy ); taus.push_back ( lastTau ); sigmas.push_back ( lastSigma ); evals.push_back ( evalCount );
    evalCount = 0;
  }
protected:
  void getTauAndUpdateDescentDir ( aol::MultiVector<double> &DescentDir, const aol::MultiVector<double> &CurrentPosition, aol::Vector<double> &Tau ) const {
    lastSigma = this->_filterWidth;
    GDType::getTauAndUpdateDescentDir ( DescentDir, CurrentPosition, Tau );
    lastTau = Tau[0];
  }
  double ArmijoLineSearchHelpFunction_evaluate ( const aol::MultiVector<double> &DescentDir, const aol::MultiVector<double> &CurrentPosition, const double TimestepWidth ) const {
    if ( TimestepWidth != 0 ) ++evalCount;
    return GDType::ArmijoLineSearchHelpFunction_evaluate ( DescentDir, CurrentPosition, TimestepWidth );
  }
};

static aol::ParameterParser* makeParser ( int maxLevel, int start, int stop, double lambda, double lambdaFactor,
                                          int maxIter, double stopEps, int resample, double sat, int minToZero ) {
  aol::ParameterParser *p = new aol::ParameterParser;
  p->addVariable ( "precisionLevel", maxLevel );
  p->addVariable ( "startLevel", start );
  p->addVariable ( "stopLevel", stop );
  p->addVariable ( "lambda", aol::strprintf ( "%.17g", lambda ).c_str() );
  p->addVariable ( "lambdaFactor", aol::strprintf ( "%.17g", lambdaFactor ).c_str() );
  p->addVariable ( "maxGDIterations", maxIter );
  p->addVariable ( "stopEpsilon", aol::strprintf ( "%.17g", stopEps ).c_str() );
  if ( resample ) p->addVariable ( "resampleInsteadOfProlongateDeformation", 1 );
  if ( sat >= 0 ) p->addVariable ( "enhanceContrastSaturationPercentage", aol::strprintf ( "%.17g", sat ).c_str() );
  p->addVariable ( "normalizeMinToZero", minToZero );
  return p;
}

// E = Edata + lambda Ereg and DE = DEdata + lambda DEreg (LinCombOp, as
// StandardRegistration::findTransformation builds them, registration.h:971-982);
// writes Edata, Ereg, E and [DE, DEdata].
template <typename EnergyType, typename VariationType>
static void energyCommand ( const qc::GridDefinition &grid, const EnergyType &Edata, const VariationType &DEdata,
                            const aol::MultiVector<RealType> &phi, RealType lambda, const char *prefix ) {
  const int N = grid.getNumberOfNodes ( );
  qc::DirichletRegularizationConfigurator<ConfType> regul ( grid );
  aol::LinCombOp<aol::MultiVector<RealType>, aol::Scalar<RealType> > E;
  E.appendReference ( Edata ); E.appendReference ( regul.getRegERef ( ), lambda );
  aol::LinCombOp<aol::MultiVector<RealType> > DE;
  DE.appendReference ( DEdata ); DE.appendReference ( regul.getRegDERef ( ), lambda );
  aol::Scalar<RealType> edata, ereg, etot;
  Edata.apply ( phi, edata ); regul.getRegERef ( ).apply ( phi, ereg ); E.apply ( phi, etot );
  aol::MultiVector<RealType> de ( 2, N ), fo ( 2, N );
  DE.apply ( phi, de );
  DEdata.apply ( phi, fo );
  std::vector<RealType> out ( 4 * N );
  memcpy ( &out[0], de[0].getData ( ), N * sizeof ( RealType ) );
  memcpy ( &out[N], de[1].getData ( ), N * sizeof ( RealType ) );
  memcpy ( &out[2 * N], fo[0].getData ( ), N * sizeof ( RealType ) );
  memcpy ( &out[3 * N], fo[1].getData ( ), N * sizeof ( RealType ) );
  writeBin ( ( std::string ( prefix ) + "_de.bin" ).c_str ( ), &out[0], 4 * N );
  FILE *f = fopen ( ( std::string ( prefix ) + ".txt" ).c_str ( ), "w" );
  fprintf ( f, "%.17g %.17g %.17g\n", edata[0], ereg[0], etot[0] );
  fclose ( f );
}

// StandardRegistration::findTransformation + updateTransformationWithGD
// (registration.h:967-1021) with the tracing solver.
template <typename EnergyType, typename VariationType>
static void gdLevelCommand ( const qc::GridDefinition &grid, const EnergyType &Edata, const VariationType &DEdata,
                             aol::MultiVector<RealType> &phi, RealType lambda, int maxIter, RealType stopEps,
                             const char *outPhi, const char *outTrace ) {
  const int N = grid.getNumberOfNodes ( );
  qc::DirichletRegularizationConfigurator<ConfType> regul ( grid );
  aol::LinCombOp<aol::MultiVector<RealType>, aol::Scalar<RealType> > E;
  E.appendReference ( Edata ); E.appendReference ( regul.getRegERef ( ), lambda );
  aol::LinCombOp<aol::MultiVector<RealType> > DE;
  DE.appendReference ( DEdata ); DE.appendReference ( regul.getRegDERef ( ), lambda );
  TracingGD gd ( grid, E, DE, maxIter, stopEps );
  gd.setConfigurationFlags ( GDType::USE_NONLINEAR_CG | GDType::DO_NOT_WRITE_CONSOLE_OUTPUT );
  gd.applySingle ( phi );
  std::vector<RealType> out ( 2 * N );
  memcpy ( &out[0], phi[0].getData ( ), N * sizeof ( RealType ) );
  memcpy ( &out[N], phi[1].getData ( ), N * sizeof ( RealType ) );
  writeBin ( outPhi, &out[0], 2 * N );
  FILE *f = fopen ( outTrace, "w" );
  fprintf ( f, "# iter energy tau sigma evals ; final %.17g steps %d\n", gd.getEnergyAtLastPosition ( ), gd.getIterations ( ) );
  for ( size_t i = 0; i < gd.energies.size ( ); ++i )
    fprintf ( f, "%d %.17g %.17g %.17g %d\n", ( int ) i, gd.energies[i], gd.taus[i], gd.sigmas[i], gd.evals[i] );
  fclose ( f );
}

// solveAndProlongToMaxDepth of the registration class Regis from a given
// displacement (registration.h:462-467).
template <typename Regis>
static void registerCommand ( char **argv ) {
  const int maxL = atoi ( argv[2] ), start = atoi ( argv[3] ), stop = atoi ( argv[4] );
  const int n = lvlN ( maxL ), N = n * n;
  aol::ParameterParser *parser = makeParser ( maxL, start, stop, atof ( argv[9] ), atof ( argv[10] ), atoi ( argv[11] ),
                                              atof ( argv[12] ), atoi ( argv[13] ), -1, 0 );
  Regis regis ( *parser );
  qc::GridDefinition grid ( maxL, qc::QC_2D );
  ArrayType R ( grid ), T ( grid );
  readBin ( argv[5], R.getData ( ), N ); readBin ( argv[6], T.getData ( ), N );
  regis.initRefOrTemplate ( R, qc::REFERENCE, true );
  regis.initRefOrTemplate ( T, qc::TEMPLATE, true );
  qc::MultiArray<RealType, qc::QC_2D> phi ( grid );
  readBin ( argv[7], phi[0].getData ( ), N ); readBin ( argv[8], phi[1].getData ( ), N );
  regis.setTransformation ( phi );
  regis.solveAndProlongToMaxDepth ( );
  regis.getTransformation ( phi );
  std::vector<RealType> out ( 2 * N );
  memcpy ( &out[0], phi[0].getData ( ), N * sizeof ( RealType ) );
  memcpy ( &out[N], phi[1].getData ( ), N * sizeof ( RealType ) );
  writeBin ( argv[14], &out[0], 2 * N );
  FILE *f = fopen ( argv[15], "w" );
  fprintf ( f, "%.17g\n", regis.getEnergyOfLastSolution ( ) );
  fclose ( f );
  delete parser;
}

// One stage of series matching with a fixed reference: every frame is
// prepared (normalised), registered to the reference from a zero
// displacement, and the raw frames are averaged after warping
// (matchSeries.h:141-155, 385-425).  Frame 0 of framesBin is the reference.
template <typename Regis>
static void seriesCommand ( char **argv ) {
  const int maxL = atoi ( argv[2] ), start = atoi ( argv[3] ), stop = atoi ( argv[4] );
  const int n = lvlN ( maxL ), N = n * n;
  const int F = atoi ( argv[11] );
  aol::ParameterParser *parser = makeParser ( maxL, start, stop, atof ( argv[5] ), atof ( argv[6] ), atoi ( argv[7] ),
                                              atof ( argv[8] ), 0, atof ( argv[9] ), atoi ( argv[10] ) );
  Regis regis ( *parser );
  qc::GridDefinition grid ( maxL, qc::QC_2D );
  std::vector<RealType> frames ( ( size_t ) N * F );
  readBin ( argv[12], &frames[0], ( size_t ) N * F );
  ArrayType ref ( grid );
  memcpy ( ref.getData ( ), &frames[0], N * sizeof ( RealType ) );
  const double t0 = wallSeconds ( );
  regis.initRefOrTemplate ( ref, qc::REFERENCE, false );
  std::vector<RealType> phis ( ( size_t ) 2 * N * F, 0. );
  std::vector<double> energies ( F, 0. );
  qc::MultiArray<RealType, qc::QC_2D> phi ( grid );
  for ( int f = 1; f < F; ++f ) {
    ArrayType tpl ( grid );
    memcpy ( tpl.getData ( ), &frames[( size_t ) f * N], N * sizeof ( RealType ) );
    regis.initRefOrTemplate ( tpl, qc::TEMPLATE, false );
    regis.setTransformationToZero ( );
    regis.solveAndProlongToMaxDepth ( );
    regis.getTransformation ( phi );
    energies[f] = regis.getEnergyOfLastSolution ( );
    memcpy ( &phis[( size_t ) 2 * f * N], phi[0].getData ( ), N * sizeof ( RealType ) );
    memcpy ( &phis[( size_t ) ( 2 * f + 1 ) * N], phi[1].getData ( ), N * sizeof ( RealType ) );
  }
  const double t1 = wallSeconds ( );
  // averageSeries: DeformImage with Inf extension, mean over finite samples.
  std::vector<RealType> mean ( N, 0. );
  {
    aol::MultiVector<RealType> deformed ( F, N );
    for ( int f = 0; f < F; ++f ) {
      aol::Vector<RealType> img ( &frames[( size_t ) f * N], N, aol::FLAT_COPY );
      aol::MultiVector<RealType> p ( 2, N );
      memcpy ( p[0].getData ( ), &phis[( size_t ) 2 * f * N], N * sizeof ( RealType ) );
      memcpy ( p[1].getData ( ), &phis[( size_t ) ( 2 * f + 1 ) * N], N * sizeof ( RealType ) );
      qc::DeformImage<ConfType> ( img, grid, deformed[f], p, true, aol::NumberTrait<RealType>::Inf, false );
    }
    aol::Vector<RealType> last ( &frames[( size_t ) ( F - 1 ) * N], N, aol::FLAT_COPY );
    const RealType lastMean = last.getMeanValue ( );
    for ( int j = 0; j < N; ++j ) {
      RealType a = 0; int k = 0;
      for ( int f = 0; f < F; ++f )
        if ( deformed[f][j] != aol::NumberTrait<RealType>::Inf ) { a += deformed[f][j]; ++k; }
      mean[j] = ( k > 0 ) ? a / k : lastMean;
    }
  }
  const double t2 = wallSeconds ( );
  writeBin ( argv[13], &phis[0], ( size_t ) 2 * N * F );
  writeBin ( argv[14], &mean[0], N );
  FILE *f = fopen ( argv[15], "w" );
  fprintf ( f, "registration_seconds %.6f\naverage_seconds %.6f\n", t1 - t0, t2 - t1 );
  for ( int i = 0; i < F; ++i ) fprintf ( f, "energy %d %.17g\n", i, energies[i] );
  fclose ( f );
  delete parser;
}

// The stage loop of matchSeries<>() (matchSeries.h:1250-1320) with the
// default options: stage 1 registers frames 1..F-1 with frame 0 as the
// reference, every further stage registers frames 0..F-1 with the average
// (or median) of the previous stage as the reference and lambda replaced by
// the "%f" print of lambda * extraStagesLambdaFactor (matchSeries.h:1300).
// Inside a stage, SeriesMatching::matchSeries (matchSeries.h:87-265) with
// accumulated deformations: each template is registered to the previous one
// from zero, its displacement is composed with the accumulated one
// (composeDeformations, registration.h:584-586) and, from the second template
// on, refined against the stage's reference on refineStartLevel..
// refineStopLevel.  The average and median of the warped raw templates follow
// averageSeries (matchSeries.h:353-445).  Writes per stage s (1-based)
// <out>_phis<s>.bin, <out>_avg<s>.bin, <out>_median<s>.bin, <out>_count<s>.bin
// and <out>.txt (energies and timings).
template <typename Regis>
static void matchSeriesCommand ( char **argv ) {
  const int maxL = atoi ( argv[2] ), start = atoi ( argv[3] ), stop = atoi ( argv[4] );
  const double lambda = atof ( argv[5] ), lamFac = atof ( argv[6] );
  const int maxIter = atoi ( argv[7] );
  const double stopEps = atof ( argv[8] ), sat = atof ( argv[9] );
  const int minToZero = atoi ( argv[10] ), refineStart = atoi ( argv[11] ), refineStop = atoi ( argv[12] );
  const int extraStages = atoi ( argv[13] );
  const double extraLamFac = atof ( argv[14] );
  const int useMedian = atoi ( argv[15] ), F = atoi ( argv[16] );
  const std::string out = argv[18];
  const int n = lvlN ( maxL ), N = n * n;
  qc::GridDefinition grid ( maxL, qc::QC_2D );
  std::vector<RealType> frames ( ( size_t ) N * F );
  readBin ( argv[17], &frames[0], ( size_t ) N * F );
  FILE *info = fopen ( ( out + ".txt" ).c_str ( ), "w" );
  ArrayType target ( grid );
  memcpy ( target.getData ( ), &frames[0], N * sizeof ( RealType ) );
  for ( int stage = 1; stage <= 1 + extraStages; ++stage ) {
    const double lam = ( stage == 1 ) ? lambda : atof ( aol::strprintf ( "%f", lambda * extraLamFac ).c_str ( ) );
    const int first = ( stage == 1 ) ? 1 : 0, m = F - first;
    aol::ParameterParser *parser = makeParser ( maxL, start, stop, lam, lamFac, maxIter, stopEps, 0, sat, minToZero );
    Regis regis ( *parser );
    const double t0 = wallSeconds ( );
    regis.initRefOrTemplate ( target, qc::REFERENCE, false );
    const ArrayType reference ( regis.getRefImageReference ( ), aol::DEEP_COPY );
    regis.setTransformationToZero ( );
    qc::MultiArray<RealType, qc::QC_2D> acc ( grid ), cur ( grid );
    regis.getTransformation ( acc );
    std::vector<RealType> phis ( ( size_t ) 2 * N * m );
    for ( int i = 0; i < m; ++i ) {
      regis.setTransformationToZero ( );
      ArrayType tpl ( grid );
      memcpy ( tpl.getData ( ), &frames[( size_t ) ( first + i ) * N], N * sizeof ( RealType ) );
      regis.initRefOrTemplate ( tpl, qc::TEMPLATE, false );
      regis.solveAndProlongToMaxDepth ( );
      double energy = regis.getEnergyOfLastSolution ( );
      regis.getTransformation ( cur );
      qc::MultiArray<RealType, qc::QC_2D> tmp ( acc, aol::DEEP_COPY );
      regis.composeDeformations ( cur, tmp, acc );
      if ( i > 0 ) {
        regis.setTransformation ( acc );
        regis.setReference ( reference );
        regis.solveAndProlongToMaxDepth ( refineStart, refineStop );
        energy = regis.getEnergyOfLastSolution ( );
        regis.getTransformation ( acc );
      }
      const qc::MultiArray<RealType, qc::QC_2D> &res = ( i == 0 ) ? cur : acc;
      memcpy ( &phis[( size_t ) 2 * i * N], res[0].getData ( ), N * sizeof ( RealType ) );
      memcpy ( &phis[( size_t ) ( 2 * i + 1 ) * N], res[1].getData ( ), N * sizeof ( RealType ) );
      fprintf ( info, "energy %d %d %.17g\n", stage, i, energy );
      regis.setReference ( regis.getTemplImageReference ( ) );
    }
    const double t1 = wallSeconds ( );
    aol::MultiVector<RealType> deformed ( m, N );
    for ( int i = 0; i < m; ++i ) {
      aol::Vector<RealType> img ( &frames[( size_t ) ( first + i ) * N], N, aol::FLAT_COPY );
      aol::MultiVector<RealType> p ( 2, N );
      memcpy ( p[0].getData ( ), &phis[( size_t ) 2 * i * N], N * sizeof ( RealType ) );
      memcpy ( p[1].getData ( ), &phis[( size_t ) ( 2 * i + 1 ) * N], N * sizeof ( RealType ) );
      qc::DeformImage<ConfType> ( img, grid, deformed[i], p, true, aol::NumberTrait<RealType>::Inf, false );
    }
    aol::Vector<RealType> last ( &frames[( size_t ) ( F - 1 ) * N], N, aol::FLAT_COPY );
    const RealType lastMean = last.getMeanValue ( );
    ArrayType avg ( grid ), cnt ( grid );
    for ( int j = 0; j < N; ++j ) {
      RealType a = 0; int k = 0;
      for ( int i = 0; i < m; ++i )
        if ( deformed[i][j] != aol::NumberTrait<RealType>::Inf ) { a += deformed[i][j]; ++k; }
      avg[j] = ( k > 0 ) ? a / k : lastMean;
      cnt[j] = k;
    }
    aol::Vector<RealType> median ( N );
    deformed.getMedianVecOverComponents ( median, lastMean );
    const double t2 = wallSeconds ( );
    fprintf ( info, "stage %d lambda %.17g registration_seconds %.6f average_seconds %.6f\n", stage, lam, t1 - t0, t2 - t1 );
    const std::string sfx = aol::strprintf ( "%d.bin", stage );
    writeBin ( ( out + "_phis" + sfx ).c_str ( ), &phis[0], ( size_t ) 2 * N * m );
    writeBin ( ( out + "_avg" + sfx ).c_str ( ), avg.getData ( ), N );
    writeBin ( ( out + "_median" + sfx ).c_str ( ), median.getData ( ), N );
    writeBin ( ( out + "_count" + sfx ).c_str ( ), cnt.getData ( ), N );
    if ( useMedian ) memcpy ( target.getData ( ), median.getData ( ), N * sizeof ( RealType ) );
    else memcpy ( target.getData ( ), avg.getData ( ), N * sizeof ( RealType ) );
    delete parser;
  }
  fclose ( info );
}

static int usage ( ) {
  fprintf ( stderr,
    "ms_ref energy[_ncc] L R T px py lambda outPrefix\n"
    "ms_ref smooth L sigma in out\n"
    "ms_ref restrict Lfine in out | prolong Lcoarse in out | resample Lsrc in Ldst out\n"
    "ms_ref deform L img px py out\n"
    "ms_ref gdlevel[_ncc] L R T px py lambda maxIter stopEps outPhi outTrace\n"
    "ms_ref register[_ncc] maxL start stop R T px py lambda lambdaFactor maxIter stopEps resample outPhi outTxt\n"
    "ms_ref normalize L in sat minToZero out\n"
    "ms_ref compose L d1 d2 inout | median L F frames phis fill out\n"
    "ms_ref save nx ny in out type | load file out dims | savedef L in mask | loaddef L mask out\n"
    "ms_ref lineshift nx ny R T phix outE outDE | xshiftreg nx ny yRegFactor phix outE outKphi\n"
    "ms_ref xshiftlap nx ny yRegFactor laplaceWeight phix outE outKphi\n"
    "ms_ref xshiftyconst nx ny maxIter R T phix outPhi outE | emptynan nx ny img out\n"
    "ms_ref rmempty nx ny keepTopBottom img out\n"
    "ms_ref h1sys nx ny sigma x out\n"
    "ms_ref series[_ncc] maxL start stop lambda lambdaFactor maxIter stopEps sat minToZero F framesBin outPhis outMean outTxt\n"
    "ms_ref matchseries[_ncc] maxL start stop lambda lambdaFactor maxIter stopEps sat minToZero refineStart refineStop\n"
    "       extraStages extraLambdaFactor useMedian F framesBin outPrefix\n" );
  return 1;
}

int main ( int argc, char **argv ) {
  if ( argc < 2 ) return usage ( );
  const std::string cmd = argv[1];
  try {
    if ( ( cmd == "energy" || cmd == "energy_ncc" ) && argc == 9 ) {
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      qc::GridDefinition grid ( L, qc::QC_2D );
      ArrayType R ( grid ), T ( grid );
      aol::MultiVector<RealType> phi ( 2, N );
      readBin ( argv[3], R.getData ( ), N ); readBin ( argv[4], T.getData ( ), N );
      readBin ( argv[5], phi[0].getData ( ), N ); readBin ( argv[6], phi[1].getData ( ), N );
      const RealType lambda = atof ( argv[7] );
      if ( cmd == "energy" ) {
        qc::SSDEnergy<ConfType> ssd ( grid, R, T );
        qc::SSDForce<ConfType> force ( grid, R, T );
        energyCommand ( grid, ssd, force, phi, lambda, argv[8] );
      } else {
        qc::NormalizedCrossCorrelationEnergy<ConfType> ncc ( grid, R, T );
        qc::VariationOfNormalizedCrossCorrelationEnergy<ConfType> var ( grid, R, T );
        energyCommand ( grid, ncc, var, phi, lambda, argv[8] );
      }
      return 0;
    }
    if ( cmd == "smooth" && argc == 6 ) {
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      qc::GridDefinition grid ( L, qc::QC_2D );
      aol::Vector<RealType> in ( N ), out ( N );
      readBin ( argv[4], in.getData ( ), N );
      qc::LinearSmoothOp<RealType> smooth ( grid );
      smooth.setSigma ( atof ( argv[3] ) );
      smooth.apply ( in, out );
      writeBin ( argv[5], out.getData ( ), N );
      return 0;
    }
    if ( cmd == "restrict" && argc == 5 ) {
      const int L = atoi ( argv[2] );
      qc::GridDefinition fine ( L, qc::QC_2D ), coarse ( L - 1, qc::QC_2D );
      aol::Vector<RealType> in ( fine.getNumberOfNodes ( ) ), out ( coarse.getNumberOfNodes ( ) );
      readBin ( argv[3], in.getData ( ), in.size ( ) );
      qc::RestrictOp<RealType, qc::STD_QUOC_RESTRICT> r ( coarse, fine );
      r.apply ( in, out );
      writeBin ( argv[4], out.getData ( ), out.size ( ) );
      return 0;
    }
    if ( cmd == "prolong" && argc == 5 ) {
      const int L = atoi ( argv[2] );
      qc::GridDefinition coarse ( L, qc::QC_2D ), fine ( L + 1, qc::QC_2D );
      aol::Vector<RealType> in ( coarse.getNumberOfNodes ( ) ), out ( fine.getNumberOfNodes ( ) );
      readBin ( argv[3], in.getData ( ), in.size ( ) );
      qc::ProlongOp<RealType> p ( coarse, fine );
      p.apply ( in, out );
      writeBin ( argv[4], out.getData ( ), out.size ( ) );
      return 0;
    }
    if ( cmd == "resample" && argc == 6 ) {
      const int Ls = atoi ( argv[2] ), Ld = atoi ( argv[4] );
      qc::GridDefinition gs ( Ls, qc::QC_2D ), gd ( Ld, qc::QC_2D );
      ArrayType src ( gs ), dst ( gd );
      readBin ( argv[3], src.getData ( ), src.size ( ) );
      dst.resampleFrom ( src );
      writeBin ( argv[5], dst.getData ( ), dst.size ( ) );
      return 0;
    }
    if ( cmd == "deform" && argc == 7 ) {
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      qc::GridDefinition grid ( L, qc::QC_2D );
      aol::Vector<RealType> img ( N ), out ( N );
      aol::MultiVector<RealType> phi ( 2, N );
      readBin ( argv[3], img.getData ( ), N );
      readBin ( argv[4], phi[0].getData ( ), N ); readBin ( argv[5], phi[1].getData ( ), N );
      qc::DeformImage<ConfType> ( img, grid, out, phi, true, aol::NumberTrait<RealType>::Inf, false );
      writeBin ( argv[6], out.getData ( ), N );
      return 0;
    }
    if ( ( cmd == "gdlevel" || cmd == "gdlevel_ncc" ) && argc == 12 ) {
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      qc::GridDefinition grid ( L, qc::QC_2D );
      ArrayType R ( grid ), T ( grid );
      aol::MultiVector<RealType> phi ( 2, N );
      readBin ( argv[3], R.getData ( ), N ); readBin ( argv[4], T.getData ( ), N );
      readBin ( argv[5], phi[0].getData ( ), N ); readBin ( argv[6], phi[1].getData ( ), N );
      const RealType lambda = atof ( argv[7] );
      const int maxIter = atoi ( argv[8] );
      const RealType stopEps = atof ( argv[9] );
      if ( cmd == "gdlevel" ) {
        qc::SSDEnergy<ConfType> ssd ( grid, R, T );
        qc::SSDForce<ConfType> force ( grid, R, T );
        gdLevelCommand ( grid, ssd, force, phi, lambda, maxIter, stopEps, argv[10], argv[11] );
      } else {
        qc::NormalizedCrossCorrelationEnergy<ConfType> ncc ( grid, R, T );
        qc::VariationOfNormalizedCrossCorrelationEnergy<ConfType> var ( grid, R, T );
        gdLevelCommand ( grid, ncc, var, phi, lambda, maxIter, stopEps, argv[10], argv[11] );
      }
      return 0;
    }
    if ( ( cmd == "register" || cmd == "register_ncc" ) && argc == 16 ) {
      if ( cmd == "register" ) registerCommand<RegisType> ( argv );
      else registerCommand<RegisTypeNCC> ( argv );
      return 0;
    }
    if ( ( cmd == "matchseries" || cmd == "matchseries_ncc" ) && argc == 19 ) {
      if ( cmd == "matchseries" ) matchSeriesCommand<RegisType> ( argv );
      else matchSeriesCommand<RegisTypeNCC> ( argv );
      return 0;
    }
    if ( cmd == "save" && argc == 7 ) {
      // ms_ref save nx ny in out type: qc::ScalarArray<QC_2D>::save (file format and compression by suffix)
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] );
      ArrayType a ( nx, ny );
      readBin ( argv[4], a.getData ( ), ( size_t ) nx * ny );
      a.save ( argv[5], static_cast<qc::SaveType> ( atoi ( argv[6] ) ) );
      return 0;
    }
    if ( cmd == "load" && argc == 5 ) {
      // ms_ref load file out dims: qc::ScalarArray<QC_2D> load, values as doubles, "numX numY" in dims
      ArrayType a ( argv[2] );
      writeBin ( argv[3], a.getData ( ), a.size ( ) );
      FILE *f = fopen ( argv[4], "w" );
      fprintf ( f, "%d %d\n", a.getNumX ( ), a.getNumY ( ) );
      fclose ( f );
      return 0;
    }
    if ( ( cmd == "savedef" || cmd == "loaddef" ) && argc == 5 ) {
      // ms_ref savedef L in mask | loaddef L mask out: qc::MultiArray save / load, one file per component
      const int L = atoi ( argv[2] ), N = lvlN ( L ) * lvlN ( L );
      qc::GridDefinition grid ( L, qc::QC_2D );
      qc::MultiArray<RealType, qc::QC_2D> phi ( grid );
      std::vector<RealType> buf ( 2 * N );
      if ( cmd == "savedef" ) {
        readBin ( argv[3], &buf[0], 2 * N );
        memcpy ( phi[0].getData ( ), &buf[0], N * sizeof ( RealType ) ); memcpy ( phi[1].getData ( ), &buf[N], N * sizeof ( RealType ) );
        phi.save ( argv[4], qc::PGM_DOUBLE_BINARY );
      } else {
        phi.load ( argv[3] );
        memcpy ( &buf[0], phi[0].getData ( ), N * sizeof ( RealType ) ); memcpy ( &buf[N], phi[1].getData ( ), N * sizeof ( RealType ) );
        writeBin ( argv[4], &buf[0], 2 * N );
      }
      return 0;
    }
    if ( cmd == "lineshift" && argc == 9 ) {
      // ms_ref lineshift nx ny R T phix outE outDE: FELineShiftRegisEnergy (registration.h:2137-2193), the data
      // term of the seismic model (matchSeismicSeries.cpp), with its derivative, on the rectangular grid
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > RectConf;
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_1D, aol::GaussQuadrature<RealType, qc::QC_1D, 3> > RectConf1D;
      typedef qc::FELineShiftRegisEnergy<RectConf, RectConf1D, qc::NCCRegistrationConfigurator<RectConf1D> > LineEnergy;
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] ), N = nx * ny;
      ArrayType R ( nx, ny ), T ( nx, ny );
      readBin ( argv[4], R.getData ( ), N ); readBin ( argv[5], T.getData ( ), N );
      const RectConf::InitType grid ( qc::GridSize<qc::QC_2D>::createFrom ( R ) );
      aol::Vector<RealType> phi ( N ), de ( N );
      readBin ( argv[6], phi.getData ( ), N );
      LineEnergy E ( grid, R, T );
      aol::Scalar<RealType> e;
      E.apply ( phi, e );
      const aol::DerivativeWrapper<RealType, LineEnergy, aol::Vector<RealType> > DE ( E );
      DE.apply ( phi, de );
      writeBin ( argv[7], &e[0], 1 );
      writeBin ( argv[8], de.getData ( ), N );
      return 0;
    }
    if ( cmd == "emptynan" && argc == 6 ) {
      // ms_ref emptynan nx ny img out: replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157), composed from the
      // same reference components (getLine, Vector::normSqr, putLine), as the function's header is not among the
      // modules
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] );
      ArrayType img ( nx, ny );
      readBin ( argv[4], img.getData ( ), nx * ny );
      qc::ScalarArray<RealType, qc::QC_1D> imageLine ( nx ), nanLine ( nx );
      nanLine.setAll ( aol::NumberTrait<RealType>::NaN );
      for ( int line = 0; line < ny; ++line ) {
        img.getLine ( qc::QC_Y, line, imageLine );
        if ( imageLine.normSqr ( ) == 0 )
          img.putLine ( qc::QC_Y, line, nanLine );
      }
      writeBin ( argv[5], img.getData ( ), nx * ny );
      return 0;
    }
    if ( cmd == "rmempty" && argc == 7 ) {
      // ms_ref rmempty nx ny keepTopBottom img out: removeEmptyLinesFromImage (matchSeismicSeries.h:101-136),
      // composed from the same reference components (getLine, normSqr, numNonNaNs, Rint, reallocate, putLine)
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] );
      const bool keep = atoi ( argv[4] ) != 0;
      ArrayType img ( nx, ny ), cleaned;
      readBin ( argv[5], img.getData ( ), nx * ny );
      qc::ScalarArray<RealType, qc::QC_1D> imageLine ( nx );
      aol::Vector<int> emptyLines, nonEmptyLines;
      for ( int line = 0; line < ny; ++line ) {
        img.getLine ( qc::QC_Y, line, imageLine );
        if ( ( imageLine.normSqr ( ) == 0 ) || ( aol::VectorHelper<aol::Vector<RealType> >::numNonNaNs ( imageLine ) == 0 ) )
          emptyLines.pushBack ( line );
        else
          nonEmptyLines.pushBack ( line );
      }
      const int first = nonEmptyLines[0], last = nonEmptyLines[nonEmptyLines.size ( ) - 1];
      const int dist = aol::Rint ( ( last - first ) / static_cast<RealType> ( nonEmptyLines.size ( ) - 1 ) );
      const int top = keep ? ( first / dist ) : 0, bottom = keep ? ( ( ny - 1 - last ) / dist ) : 0;
      cleaned.reallocate ( nx, nonEmptyLines.size ( ) + top + bottom );
      for ( int line = 0; line < nonEmptyLines.size ( ); ++line ) {
        img.getLine ( qc::QC_Y, nonEmptyLines[line], imageLine );
        cleaned.putLine ( qc::QC_Y, line + top, imageLine );
      }
      writeBin ( argv[6], cleaned.getData ( ), cleaned.size ( ) );
      return 0;
    }
    if ( cmd == "xshiftyconst" && argc == 10 ) {
      // ms_ref xshiftyconst nx ny maxIter R T phix outPhi outE: findXShiftYConst (matchSeries.h:873-920), composed
      // from the same reference components in the same order (the function's header is not among the modules)
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > RectConf;
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_1D, aol::GaussQuadrature<RealType, qc::QC_1D, 3> > RectConf1D;
      typedef qc::FELineShiftRegisEnergy<RectConf, RectConf1D, qc::NCCRegistrationConfigurator<RectConf1D> > LineEnergy;
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] ), maxIter = atoi ( argv[4] ), N = nx * ny;
      ArrayType R ( nx, ny ), T ( nx, ny ), PhiX ( nx, ny );
      readBin ( argv[5], R.getData ( ), N ); readBin ( argv[6], T.getData ( ), N );
      readBin ( argv[7], PhiX.getData ( ), N );
      const RectConf::InitType grid ( qc::GridSize<qc::QC_2D>::createFrom ( R ) );
      ArrayType temSmoothed ( grid );
      aol::Vector<RealType> tmp ( grid.getNumY() );
      PhiX.sumInXDirectionTo ( tmp );
      tmp /= grid.getNumX();
      RealType energyVal = aol::NumberTrait<RealType>::Inf;
      for ( int i = 3; i >= 0; --i ) {
        if ( i > 0 ) {
          qc::ModifiableKernel2d<RealType> xAveraginKernel ( 4 * i + 1 );
          const int offset = xAveraginKernel.getOffset();
          for ( int X = -offset; X <= offset; X++ )
            xAveraginKernel.setValue ( X, 0, 1. / ( 2 * offset + 1 ) );
          T.applyLinearFilterTo ( xAveraginKernel, temSmoothed );
        } else
          temSmoothed = T;
        const LineEnergy EData ( grid, R, temSmoothed );
        const aol::DerivativeWrapper<RealType, LineEnergy, aol::Vector<RealType> > DEData ( EData );
        const qc::PixelWiseToRowWiseOp<RectConf> E ( grid, EData, DEData );
        const aol::DerivativeWrapper<RealType, qc::PixelWiseToRowWiseOp<RectConf>, aol::Vector<RealType> > DE ( E );
        typedef aol::GridlessGradientDescent<RealType, aol::Vector<RealType> > GDType;
        GDType gdSolver ( grid, E, DE, maxIter );
        gdSolver.setConfigurationFlags ( GDType::USE_NONLINEAR_CG );
        gdSolver.applySingle ( tmp );
        energyVal = gdSolver.getEnergyAtLastPosition();
      }
      PhiX.setInXDirectionFrom ( tmp );
      writeBin ( argv[8], PhiX.getData ( ), N );
      writeBin ( argv[9], &energyVal, 1 );
      return 0;
    }
    if ( cmd == "xshiftlap" && argc == 9 ) {
      // ms_ref xshiftlap nx ny yRegFactor laplaceWeight phix outE outKphi: the regulariser of findXShift with
      // laplaceWeight > 0 (matchSeries.h:828-838): laplaceWeight L M^-1 L + stiffX + yRegFactor stiffY as CSR
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > RectConf;
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] ), N = nx * ny;
      ArrayType dummy ( nx, ny );
      const RectConf::InitType grid ( qc::GridSize<qc::QC_2D>::createFrom ( dummy ) );
      const aol::FEOpMixedDerivative<RectConf> stiffX ( grid, 0, 0, aol::ONTHEFLY );
      const aol::FEOpMixedDerivative<RectConf> stiffY ( grid, 1, 1, aol::ONTHEFLY );
      aol::SparseMatrix<RealType> tempMat ( grid );
      qc::assembleLaplaceSquareRegMatrix<RectConf> ( grid, tempMat );
      tempMat *= atof ( argv[5] );
      stiffX.assembleAddMatrix ( tempMat );
      stiffY.assembleAddMatrix ( tempMat, atof ( argv[4] ) );
      const aol::CSR_Matrix<> K ( tempMat );
      const aol::QuadraticFormOp<aol::Vector<RealType> > EReg ( K );
      aol::Vector<RealType> phi ( N ), kphi ( N );
      readBin ( argv[6], phi.getData ( ), N );
      aol::Scalar<RealType> e;
      EReg.apply ( phi, e );
      K.apply ( phi, kphi );
      writeBin ( argv[7], &e[0], 1 );
      writeBin ( argv[8], kphi.getData ( ), N );
      return 0;
    }
    if ( cmd == "xshiftreg" && argc == 8 ) {
      // ms_ref xshiftreg nx ny yRegFactor phix outE outKphi: the regulariser of findXShift with laplaceWeight <= 0
      // (matchSeries.h:819-845): K = stiffX + yRegFactor * stiffY assembled, E = 1/2 phi.K phi, and K phi
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > RectConf;
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] ), N = nx * ny;
      ArrayType dummy ( nx, ny );
      const RectConf::InitType grid ( qc::GridSize<qc::QC_2D>::createFrom ( dummy ) );
      const aol::FEOpMixedDerivative<RectConf> stiffX ( grid, 0, 0, aol::ONTHEFLY );
      const aol::FEOpMixedDerivative<RectConf> stiffY ( grid, 1, 1, aol::ONTHEFLY );
      RectConf::MatrixType K ( grid );
      stiffX.assembleAddMatrix ( K );
      stiffY.assembleAddMatrix ( K, atof ( argv[4] ) );
      const aol::QuadraticFormOp<aol::Vector<RealType> > EReg ( K );
      aol::Vector<RealType> phi ( N ), kphi ( N );
      readBin ( argv[5], phi.getData ( ), N );
      aol::Scalar<RealType> e;
      EReg.apply ( phi, e );
      K.apply ( phi, kphi );
      writeBin ( argv[6], &e[0], 1 );
      writeBin ( argv[7], kphi.getData ( ), N );
      return 0;
    }
    if ( cmd == "h1sys" && argc == 7 ) {
      // ms_ref h1sys nx ny sigma x out: the system matrix of InverseH1MetricBase (linearSmoothOp.h:262-301),
      // M + tau L with tau = 0.5f * sigma^2, assembled on the rectangular grid, applied to x.  (Its Cholesky
      // inverse, CholeskyBasedInverseH1Metric, needs SuiteSparse, which the reference does not vendor.)
      typedef qc::RectangularGridConfigurator<RealType, qc::QC_2D, aol::GaussQuadrature<RealType, qc::QC_2D, 3> > RectConf;
      const int nx = atoi ( argv[2] ), ny = atoi ( argv[3] ), N = nx * ny;
      ArrayType dummy ( nx, ny );
      const RectConf::InitType grid ( qc::GridSize<qc::QC_2D>::createFrom ( dummy ) );
      const aol::MassOp<RectConf> massOp ( grid );
      const aol::StiffOp<RectConf> stiffOp ( grid );
      RectConf::MatrixType sys ( grid );
      const RealType sigma = atof ( argv[4] );
      const RealType tau = 0.5f * aol::Sqr ( sigma );
      sys.setZero ( );
      massOp.assembleAddMatrix ( sys );
      stiffOp.assembleAddMatrix ( sys, tau );
      aol::Vector<RealType> x ( N ), y ( N );
      readBin ( argv[5], x.getData ( ), N );
      sys.apply ( x, y );
      writeBin ( argv[6], y.getData ( ), N );
      return 0;
    }
    if ( cmd == "compose" && argc == 7 ) {
      // ms_ref compose L d1 d2 inout (2 components each; inout: initial guess in, result out)
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      qc::GridDefinition grid ( L, qc::QC_2D );
      aol::MultiVector<RealType> d1 ( 2, N ), d2 ( 2, N ), out ( 2, N );
      std::vector<RealType> buf ( 2 * N );
      readBin ( argv[3], &buf[0], 2 * N );
      memcpy ( d1[0].getData ( ), &buf[0], N * sizeof ( RealType ) ); memcpy ( d1[1].getData ( ), &buf[N], N * sizeof ( RealType ) );
      readBin ( argv[4], &buf[0], 2 * N );
      memcpy ( d2[0].getData ( ), &buf[0], N * sizeof ( RealType ) ); memcpy ( d2[1].getData ( ), &buf[N], N * sizeof ( RealType ) );
      readBin ( argv[5], &buf[0], 2 * N );
      memcpy ( out[0].getData ( ), &buf[0], N * sizeof ( RealType ) ); memcpy ( out[1].getData ( ), &buf[N], N * sizeof ( RealType ) );
      qc::ConcatAndSmoothlyExtendDeformations<ConfType> ( d1, d2, grid, out );
      memcpy ( &buf[0], out[0].getData ( ), N * sizeof ( RealType ) ); memcpy ( &buf[N], out[1].getData ( ), N * sizeof ( RealType ) );
      writeBin ( argv[6], &buf[0], 2 * N );
      return 0;
    }
    if ( cmd == "median" && argc == 8 ) {
      // ms_ref median L F frames phis fill out: median of the warped frames (Inf extension)
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n, F = atoi ( argv[3] );
      qc::GridDefinition grid ( L, qc::QC_2D );
      std::vector<RealType> frames ( ( size_t ) F * N ), phis ( ( size_t ) 2 * F * N );
      readBin ( argv[4], &frames[0], ( size_t ) F * N );
      readBin ( argv[5], &phis[0], ( size_t ) 2 * F * N );
      aol::MultiVector<RealType> deformed ( F, N );
      for ( int f = 0; f < F; ++f ) {
        aol::Vector<RealType> img ( &frames[( size_t ) f * N], N, aol::FLAT_COPY );
        aol::MultiVector<RealType> p ( 2, N );
        memcpy ( p[0].getData ( ), &phis[( size_t ) 2 * f * N], N * sizeof ( RealType ) );
        memcpy ( p[1].getData ( ), &phis[( size_t ) ( 2 * f + 1 ) * N], N * sizeof ( RealType ) );
        qc::DeformImage<ConfType> ( img, grid, deformed[f], p, true, aol::NumberTrait<RealType>::Inf, false );
      }
      aol::Vector<RealType> median ( N );
      deformed.getMedianVecOverComponents ( median, atof ( argv[6] ) );
      writeBin ( argv[7], median.getData ( ), N );
      return 0;
    }
    if ( cmd == "normalize" && argc == 7 ) {
      const int L = atoi ( argv[2] ), n = lvlN ( L ), N = n * n;
      aol::ParameterParser *parser = makeParser ( L, L, L, 1, 1, 1, 0, 0, atof ( argv[4] ), atoi ( argv[5] ) );
      RegisType regis ( *parser );
      qc::GridDefinition grid ( L, qc::QC_2D );
      ArrayType img ( grid );
      readBin ( argv[3], img.getData ( ), N );
      regis.initRefOrTemplate ( img, qc::REFERENCE, false );
      writeBin ( argv[6], regis.getRefImageReference ( ).getData ( ), N );
      delete parser;
      return 0;
    }
    if ( ( cmd == "series" || cmd == "series_ncc" ) && argc == 16 ) {
      if ( cmd == "series" ) seriesCommand<RegisType> ( argv );
      else seriesCommand<RegisTypeNCC> ( argv );
      return 0;
    }
  } catch ( aol::Exception &e ) {
    e.dump ( );
    return 3;
  }
  return usage ( );
}
