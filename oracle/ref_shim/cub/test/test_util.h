// Stand-in for cub/test/test_util.h of CUB 1.6.4, which the reference's drivers
// include for CommandLineArgs (src/ssb-jo/q33/0-lip.cu:10,310-325) but which CUDA
// 12.9's bundled CUB no longer ships.  Only the three members the drivers call.
// TEST INFRASTRUCTURE: used only to compile the reference into oracle/_ref.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

struct CommandLineArgs {
  std::vector<std::string> keys, values;
  CommandLineArgs(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i];
      if (a.rfind("--", 0) != 0) continue;
      a = a.substr(2);
      const size_t eq = a.find('=');
      keys.push_back(a.substr(0, eq));
      values.push_back(eq == std::string::npos ? std::string() : a.substr(eq + 1));
    }
  }
  bool CheckCmdLineFlag(const char* name) const {
    for (const auto& k : keys)
      if (k == name) return true;
    return false;
  }
  template <typename T>
  void GetCmdLineArgument(const char* name, T& val) const {
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i] == name) {
        std::istringstream s(values[i]);
        s >> val;
      }
  }
  cudaError_t DeviceInit(int dev = -1) {
    if (dev < 0) {
      dev = 0;
      GetCmdLineArgument("device", dev);
    }
    return cudaSetDevice(dev);
  }
};
