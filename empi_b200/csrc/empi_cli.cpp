// empi-gpu: drop-in for the empi CLI (src/empi.cpp:169-195).  Takes one config
// file path; arguments starting with '-' are ignored for MP5 compatibility;
// errors print "ERROR\t<message>" on stdout and exit with status 1.
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "../../include/empi_b200.h"

int main(int argc, char** argv) {
    const char* config = nullptr;
    for (int i = 1; i < argc; ++i)
        if (*argv[i] != '-' && *argv[i] != 0) config = argv[i];
    if (!config) {
        fprintf(stderr, "USAGE: %s path_to_config_file\n", argv[0]);
        return 1;
    }
    empi_engine_opts opts;
    empi_engine_opts_default(&opts);
    if (const char* dev = getenv("EMPI_DEVICE")) opts.device = atoi(dev);
    empi_status st = empi_run_config(config, &opts);
    if (st != EMPI_OK) {
        std::cout << "ERROR\t" << empi_last_error() << std::endl;
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}
