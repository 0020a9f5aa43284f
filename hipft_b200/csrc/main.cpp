// main.cpp -- `hipft [hipft.in]`, the standalone executable
// (command line of src/hipft.f90:8416-8423): runs in the current directory.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/hipft_gpu.h"

int main(int argc, char **argv) {
  std::string in = argc > 1 ? argv[1] : "hipft.in";
  const char *dev = std::getenv("HIPFT_DEVICE");
  int rc = hipft_run(in.c_str(), ".", dev ? std::atoi(dev) : 0);
  return rc == HIPFT_OK ? 0 : 1;
}
