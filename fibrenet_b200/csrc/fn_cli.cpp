/*
 * fn_cli.cpp -- non-interactive replacement of FibreNet.cpp's _tmain
 * (FibreNet/FibreNet.cpp:6-15): the input file and device come from the
 * command line instead of std::cin and the OpenCL platform prompts.
 *
 *     fibrenet_run <input_file> [--device N] [--strict]
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/fibrenet_io.h"

int main(int argc, char** argv) {
    const char* input = nullptr;
    int device = 0, strict = 0;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--strict"))
            strict = 1;
        else if (!input)
            input = argv[i];
        else {
            std::fprintf(stderr, "usage: %s <input_file> [--device N] [--strict]\n", argv[0]);
            return 2;
        }
    }
    if (!input) {
        std::fprintf(stderr, "usage: %s <input_file> [--device N] [--strict]\n", argv[0]);
        return 2;
    }
    char err[512] = {0};
    const int rc = fn_run_input(input, device, strict, err, sizeof err);
    if (rc != 0) {
        std::fprintf(stderr, "fibrenet_run: %s (status %d)\n", err, rc);
        return 1;
    }
    std::fprintf(stderr, "fibrenet_run: finished\n");
    return 0;
}
