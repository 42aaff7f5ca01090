// clast_cli.cpp -- `clast` binary: the reference's command line on the GPU.
#include <cstdio>

#include "clast_host.h"

int main(int argc, const char** argv) {
  char err[1024] = {0};
  const int rc = clast_cli_main(argc, argv, err, sizeof(err));
  if (rc != 0) std::fprintf(stderr, " error : %s\n", err);
  return rc;
}
