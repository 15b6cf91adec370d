/* Test infrastructure: <direct.h> names come from win32_compat.h. */
