// Drop-in executable for the reference's main (main.cpp:6-9):
//   qmcrt -c config.json -s scene.scn -h heliostat_index.txt -o output_dir/
#include "qmcrt.h"

int main(int argc, char** argv) { return qmcrt_pipeline_run(argc, argv); }
