/* Test infrastructure: <psapi.h> content is provided by the windows.h stand-in. */
#include "windows.h"
