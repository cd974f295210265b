// Drop-in GraphWalker API: the one include of every app
// (the reference's src/api/graphwalker_basic_includes.hpp).
#ifndef GRAPHWALKER_DEF_ALLBASIC_INCLUDES
#define GRAPHWALKER_DEF_ALLBASIC_INCLUDES

#include <omp.h>

#include <cstring>
#include <sstream>

#include "api/cmdopts.hpp"
#include "api/filename.hpp"
#include "engine/graphwalker.hpp"
#include "logger/logger.hpp"
#include "metrics/metrics.hpp"
#include "metrics/reps/basic_reporter.hpp"
#include "metrics/reps/file_reporter.hpp"
#include "metrics/reps/html_reporter.hpp"
#include "preprocess/conversions.hpp"

// Console report and the graphwalker_metrics.txt file report (with its
// .statistics row), as the reference's metrics_report does.
static VARIABLE_IS_NOT_USED void metrics_report(metrics& m) {
  basic_reporter console;
  m.report(console);
  file_reporter file(get_option_string("metrics.reporter.filename", "graphwalker_metrics.txt"));
  m.report(file);
}

#endif
