#ifndef DCA_CONFIG_THREADING_DEFINES_HPP
#define DCA_CONFIG_THREADING_DEFINES_HPP
#include "dca/config/haves_defines.hpp"
#include "dca/config/config_defines.hpp"
#include "dca/parallel/stdthread/stdthread.hpp"
#include "dca/parallel/stdthread/thread_pool/affinity.hpp"
using Threading = dca::parallel::stdthread;
#endif
