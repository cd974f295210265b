// Drop-in GraphWalker API: key=value configuration files
// (the reference's src/api/configfile.hpp:81-117: '#' and '%' lines are
// comments, keys and values are trimmed, the secondary file is read when the
// primary one is absent, and having neither is fatal).
#ifndef GRAPHCHI_CONFIGFILE_DEF
#define GRAPHCHI_CONFIGFILE_DEF

#include <cassert>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <map>
#include <string>

static inline std::string gw_trim(std::string s) {
  const char* ws = " \f\n\r\t\v";
  const size_t b = s.find_first_not_of(ws);
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(ws);
  return s.substr(b, e - b + 1);
}

static inline std::map<std::string, std::string> loadconfig(std::string filename,
                                                            std::string secondary_filename) {
  FILE* f = fopen(filename.c_str(), "r");
  if (!f) {
    f = fopen(secondary_filename.c_str(), "r");
    if (!f) {
      std::cout << "ERROR: Could not read configuration file: " << filename << std::endl;
      std::cout << "Please define environment variable GRAPHCHI_ROOT or run the program from that directory."
                << std::endl;
    }
    assert(f != NULL);
    if (!f) abort();
  }
  std::map<std::string, std::string> conf;
  char line[4096];
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '%') continue;
    std::string s(line);
    const size_t eq = s.find('=');
    if (eq == std::string::npos) continue;
    std::string key = gw_trim(s.substr(0, eq)), val = gw_trim(s.substr(eq + 1));
    const size_t eq2 = val.find('=');  // the reference tokenises on '=': a value ends at the next one
    if (eq2 != std::string::npos) val = gw_trim(val.substr(0, eq2));
    if (!key.empty() && !val.empty()) conf[key] = val;
  }
  fclose(f);
  return conf;
}

#endif
