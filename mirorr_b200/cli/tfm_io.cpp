// tfm_io.cpp -- ITK transform file reader / writer (see tfm_io.hpp).
#include "tfm_io.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <vector>

namespace mirorr_cli {

mirorr_transform read_tfm(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  mirorr_transform t;
  std::memset(&t, 0, sizeof(t));
  t.kind = -1;
  std::vector<double> params, fixed;
  std::string line;
  while (std::getline(in, line)) {
    if (line.rfind("Transform:", 0) == 0) {
      if (t.kind >= 0) break;  // the first transform of the file
      if (line.find("Euler3DTransform") != std::string::npos) t.kind = 0;
      else if (line.find("AffineTransform") != std::string::npos) t.kind = 1;
      else throw std::runtime_error("unsupported transform type in " + path + ": " + line);
    } else if (line.rfind("Parameters:", 0) == 0) {
      std::istringstream s(line.substr(11));
      double v;
      while (s >> v) params.push_back(v);
    } else if (line.rfind("FixedParameters:", 0) == 0) {
      std::istringstream s(line.substr(16));
      double v;
      while (s >> v) fixed.push_back(v);
    }
  }
  if (t.kind < 0) throw std::runtime_error("no transform in " + path);
  const size_t np = t.kind == 0 ? 6 : 12;
  if (params.size() != np || fixed.size() < 3)
    throw std::runtime_error("malformed transform parameters in " + path);
  for (size_t i = 0; i < np; ++i) t.params[i] = params[i];
  for (int i = 0; i < 3; ++i) t.center[i] = fixed[i];
  return t;
}

void write_tfm(const std::string &path, const mirorr_transform &t) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write " + path);
  const int np = t.kind == 0 ? 6 : 12;
  std::fprintf(f, "#Insight Transform File V1.0\n#Transform 0\nTransform: %s\nParameters:",
               t.kind == 0 ? "Euler3DTransform_double_3_3" : "AffineTransform_double_3_3");
  for (int i = 0; i < np; ++i) std::fprintf(f, " %.17g", t.params[i]);
  std::fprintf(f, "\nFixedParameters:");
  for (int i = 0; i < 3; ++i) std::fprintf(f, " %.17g", t.center[i]);
  std::fprintf(f, "\n");
  if (std::fclose(f) != 0) throw std::runtime_error("write failed: " + path);
}

}  // namespace mirorr_cli
