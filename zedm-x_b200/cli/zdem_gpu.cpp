// zdem_gpu -- drop-in for zdem_cpu (src/main.cpp:1691-1708, 1872-1881): `zdem_gpu --config file.txt`.
// Same arguments, exit codes, outputs and log line; the step runs on the GPU through libzdemx.so.
#include <cstdlib>
#include <iostream>
#include <string>

#include "../../include/zdemx.h"

static bool parse_args(int argc, char** argv, std::string& config_path) {
    for (int i = 1; i < argc; ++i) {
        std::string arg = argv[i];
        if (arg == "--config" && i + 1 < argc) {
            config_path = argv[++i];
        } else if (arg == "--help") {
            return false;
        } else {
            std::cerr << "Unknown arg: " << arg << "\n";
            return false;
        }
    }
    return !config_path.empty();
}

int main(int argc, char** argv) {
    std::string config_path;
    if (!parse_args(argc, argv, config_path)) {
        std::cout << "Usage: zdem_gpu --config path.txt\n";
        return 1;
    }
    const char* dev = std::getenv("ZDEMX_DEVICE");
    return zdx_run_config(config_path.c_str(), dev ? std::atoi(dev) : 0);
}
