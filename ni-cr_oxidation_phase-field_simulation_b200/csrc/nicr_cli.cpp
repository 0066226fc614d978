// The solver programs nicr2d / nicr3d: the reference's executables
// (2D:1248-1254, 3S:1397-1403) as thin mains over the C-ABI.
#include "../../include/nicr.h"

int main(int argc, char** argv) { return nicr_main(NICR_CLI_DIM, argc, (const char* const*)argv); }
