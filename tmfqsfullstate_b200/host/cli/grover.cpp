#include "grover_cli.h"

int main(int argc, char *argv[]) { return tmfqs_cli::runGroverCli(argc, argv, "grover", "normal", true); }
