// zdem_gpu -- drop-in for zdem_cpu (src/main.cpp:1691-1708, 1872-1881): `zdem_gpu --config file.txt`.
// Same arguments, exit codes, outputs and log line; the step runs on the GPU through libzdemx.so.
// `--graph` (an addition) runs the steps between outputs as one captured CUDA graph each.
#include <cstdlib>
#include <iostream>
#include <string>

#include "../../include/zdemx.h"

static bool parse_args(int argc, char** argv, std::string& config_path, bool& graph) {
    for (int i = 1; i < argc; ++i) {
        std::string arg = argv[i];
        if (arg == "--config" && i + 1 < argc) {
            config_path = argv[++i];
        } else if (arg == "--graph") {
            graph = true;
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
    bool graph = false;
    if (!parse_args(argc, argv, config_path, graph)) {
        std::cout << "Usage: zdem_gpu --config path.txt [--graph]\n";
        return 1;
    }
    const char* dev = std::getenv("ZDEMX_DEVICE");
    const int d = dev ? std::atoi(dev) : 0;
    return graph ? zdx_run_config_graph(config_path.c_str(), d) : zdx_run_config(config_path.c_str(), d);
}
