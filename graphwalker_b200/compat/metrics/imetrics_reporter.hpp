// Drop-in GraphWalker API: the reporter interface lives in metrics.hpp.
#ifndef GW_COMPAT_IMETRICS_REPORTER_HPP
#define GW_COMPAT_IMETRICS_REPORTER_HPP
#include "metrics/metrics.hpp"
#endif
