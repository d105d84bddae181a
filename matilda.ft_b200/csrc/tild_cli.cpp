// tild_cli.cpp -- `tild_run [-in file] [-device k]`, the command-line driver that takes
// the place of MATILDA.FT's `matilda.ft` executable (main.cu:21-156) for PS boxes.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "tild_b200.h"

int main(int argc, char **argv)
{
    std::string input = "input";   // main.cu:35
    int device = 0;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "-in" && i + 1 < argc) {
            input = argv[++i];
        } else if (a == "-device" && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else {
            std::fprintf(stderr, "%s is not a valid argument\n", a.c_str());
            return 1;
        }
    }
    const int rc = tild_run_script_file(input.c_str(), device);
    if (rc != TILD_OK) {
        std::fprintf(stderr, "tild_run: error %d: %s\n", rc, tild_last_error());
        return 1;
    }
    return 0;
}
