#ifndef DCA_PHYS_DCA_DATA_DCA_DATA_HPP
#define DCA_PHYS_DCA_DATA_DCA_DATA_HPP
#include <complex>
#include "dca/distribution/dist_types.hpp"
#include "dca/function/domains.hpp"
#include "dca/function/function.hpp"
#include "dca/phys/domains/cluster/momentum_exchange_domain.hpp"
#include "dca/phys/domains/quantum/electron_band_domain.hpp"
#include "dca/phys/domains/time_and_frequency/frequency_exchange_domain.hpp"
#include "dca/phys/domains/time_and_frequency/vertex_frequency_domain.hpp"
namespace dca { namespace phys {
template <class Parameters, DistType DIST = DistType::NONE>
class DcaData {
public:
  using TpComplex = std::complex<typename Parameters::TPAccumPrec>;
  using WVertexDmn = func::dmn_0<domains::vertex_frequency_domain<domains::COMPACT>>;
  using WExchangeDmn = func::dmn_0<domains::FrequencyExchangeDomain>;
  using BDmn = func::dmn_0<domains::electron_band_domain>;
  using KClusterDmn = typename Parameters::KClusterDmn;
  using KExchangeDmn = func::dmn_0<domains::MomentumExchangeDomain>;
  using TpGreensFunction =
      func::function<TpComplex, func::dmn_variadic<BDmn, BDmn, BDmn, BDmn, KClusterDmn, WVertexDmn,
                                                   KClusterDmn, WVertexDmn, KExchangeDmn, WExchangeDmn>,
                     DIST>;
};
}}
#endif
