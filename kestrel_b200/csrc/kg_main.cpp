// kestrel — command-line entry point; see kg_run_cli in kg_cli.cpp.
#include "kestrel_gpu.h"

int main(int argc, char** argv) { return kg_run_cli(argc, (const char* const*)argv); }
