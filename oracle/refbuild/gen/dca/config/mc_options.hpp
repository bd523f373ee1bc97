#ifndef DCA_CONFIG_MC_OPTIONS_HPP
#define DCA_CONFIG_MC_OPTIONS_HPP
namespace dca { namespace config {
struct McOptions { using MC_REAL = double; using TPAccumulationPrecision = double; static constexpr bool memory_savings = false; };
}}
#endif
