// The SOSR app: apps/SOSR.cu of GOWalker, same flags, walks on the B200
// engine through libgowalker.so.
#include "gowalker_host.hpp"

int main(int argc, const char *argv[]) { return walk_app_main(argc, argv, SOSR); }
