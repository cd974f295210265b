// Drop-in GraphWalker API: named timers and counters.
// Interface of the reference's src/metrics/metrics.hpp:162-335 (start_time /
// stop_time / set / add / report); thread-safe here, unlike the reference's
// timers, which several OpenMP threads start and stop concurrently.
#ifndef DEF_METRICS_HPP
#define DEF_METRICS_HPP

#include <sys/time.h>

#include <cfloat>
#include <map>
#include <mutex>
#include <string>
#include <vector>

enum metrictype { REAL, INTEGER, TIME, STRING, VECTOR };

struct metrics_entry {
  double value = 0, sum = 0, minvalue = DBL_MAX, maxvalue = -DBL_MAX, cumvalue = 0, lasttime = 0;
  size_t count = 0;
  metrictype valtype = REAL;
  std::string stringval;
  std::vector<double> v;
  timeval start_tv{};

  metrics_entry() {}
  metrics_entry(double firstvalue, metrictype t) : valtype(t) { add(firstvalue); value = firstvalue; }
  explicit metrics_entry(std::string s) : valtype(STRING), stringval(s) {}
  explicit metrics_entry(metrictype t) : valtype(t) {}

  void add(double x) {
    value += x;
    cumvalue += x;
    ++count;
    if (x < minvalue) minvalue = x;
    if (x > maxvalue) maxvalue = x;
  }
  void set(double x) {
    value = x;
    if (x < minvalue) minvalue = x;
    if (x > maxvalue) maxvalue = x;
  }
  void set(std::string s) { stringval = s; }
  void add_vector_entry(size_t i, double x) {
    if (v.size() <= i) v.resize(i + 1);
    v[i] += x;
  }
  void set_vector_entry(size_t i, double x) {
    if (v.size() <= i) v.resize(i + 1);
    v[i] = x;
  }
  void timer_start() { gettimeofday(&start_tv, nullptr); }
  void timer_stop() {
    timeval now;
    gettimeofday(&now, nullptr);
    lasttime = (now.tv_sec - start_tv.tv_sec) + (now.tv_usec - start_tv.tv_usec) * 1e-6;
    add(lasttime);
  }
};

class imetrics_reporter {
 public:
  virtual ~imetrics_reporter() {}
  virtual void do_report(std::string name, std::string id, std::map<std::string, metrics_entry>& entries) = 0;
};

class metrics {
  std::string name, ident;
  std::map<std::string, metrics_entry> entries;
  std::mutex mlock;

 public:
  metrics(std::string _name = "", std::string _id = "") : name(_name), ident(_id) { set("app", _name); }

  void clear() {
    std::lock_guard<std::mutex> g(mlock);
    entries.clear();
  }
  void add(std::string key, double value, metrictype type = REAL) {
    std::lock_guard<std::mutex> g(mlock);
    auto it = entries.find(key);
    if (it == entries.end()) entries[key] = metrics_entry(value, type);
    else it->second.add(value);
  }
  void add_to_vector(std::string key, double value) { add(key, value, VECTOR); }
  void add_vector_entry(std::string key, size_t idx, double value) {
    std::lock_guard<std::mutex> g(mlock);
    auto& e = entries[key];
    e.valtype = VECTOR;
    e.add_vector_entry(idx, value);
  }
  void set(std::string key, size_t value) { set(key, (double)value, INTEGER); }
  void set(std::string key, int value) { set(key, (double)value, INTEGER); }
  void set(std::string key, double value, metrictype type = REAL) {
    std::lock_guard<std::mutex> g(mlock);
    auto it = entries.find(key);
    if (it == entries.end()) entries[key] = metrics_entry(value, type);
    else it->second.set(value);
  }
  void set_integer(std::string key, size_t value) { set(key, (double)value, INTEGER); }
  void set(std::string key, std::string s) {
    std::lock_guard<std::mutex> g(mlock);
    auto it = entries.find(key);
    if (it == entries.end()) entries[key] = metrics_entry(s);
    else it->second.set(s);
  }
  void set_vector_entry_integer(std::string key, size_t idx, size_t value) { set_vector_entry(key, idx, (double)value); }
  void set_vector_entry(std::string key, size_t idx, double value) {
    std::lock_guard<std::mutex> g(mlock);
    auto& e = entries[key];
    e.valtype = VECTOR;
    e.set_vector_entry(idx, value);
  }
  void start_time(std::string key) {
    std::lock_guard<std::mutex> g(mlock);
    auto it = entries.find(key);
    if (it == entries.end()) it = entries.emplace(key, metrics_entry(TIME)).first;
    it->second.timer_start();
  }
  metrics_entry start_time() {
    metrics_entry me(TIME);
    me.timer_start();
    return me;
  }
  void stop_time(metrics_entry me, std::string key, bool show = false) {
    me.timer_stop();
    add(key, me.lasttime, TIME);
    if (show) printf("%s: %f secs.\n", key.c_str(), me.lasttime);
  }
  void stop_time(std::string key, bool show = false) {
    std::lock_guard<std::mutex> g(mlock);
    auto& e = entries[key];
    e.valtype = TIME;
    e.timer_stop();
    if (show) printf("%s: %f secs.\n", key.c_str(), e.lasttime);
  }
  // Adds a duration measured elsewhere (device time) under a timer key.
  void add_time(std::string key, double seconds) { add(key, seconds, TIME); }
  metrics_entry get(std::string key) {
    std::lock_guard<std::mutex> g(mlock);
    return entries[key];
  }
  void report(imetrics_reporter& reporter) {
    if (name != "") reporter.do_report(name, ident, entries);
  }
};

#endif
