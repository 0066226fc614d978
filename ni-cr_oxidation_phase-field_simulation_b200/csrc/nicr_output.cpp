// Output writers (placeholder until the writers land).
#include "../../include/nicr.h"
extern "C" {
int nicr_write_vtk(nicr_handle*, const char*) { return NICR_ERR_STATE; }
int nicr_write_vti(nicr_handle*, const char*) { return NICR_ERR_STATE; }
int nicr_write_metadata(nicr_handle*, const char*) { return NICR_ERR_STATE; }
int nicr_format_log_row(nicr_handle*, int, char*, size_t) { return NICR_ERR_STATE; }
int nicr_format_grain_rows(nicr_handle*, int, char*, size_t, char*, size_t) { return NICR_ERR_STATE; }
int nicr_main(int, int, const char* const*) { return 1; }
}
