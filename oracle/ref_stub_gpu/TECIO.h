/* The host-build stub of the TecIO header: file output is not part of the measured step. */
#include "../ref_stub/TECIO.h"
