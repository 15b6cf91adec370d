/* Test infrastructure: empty stand-in for <windows.h> so the reference
 * sources compile on Linux; the process-memory report becomes a no-op. */
#ifndef TDBEM_ORACLE_WINDOWS_H
#define TDBEM_ORACLE_WINDOWS_H
typedef void* HANDLE;
typedef unsigned long DWORD;
typedef struct { size_t WorkingSetSize; size_t PeakWorkingSetSize; size_t PagefileUsage; size_t PeakPagefileUsage; } PROCESS_MEMORY_COUNTERS;
static inline HANDLE GetCurrentProcess(void) { return 0; }
static inline int GetProcessMemoryInfo(HANDLE h, PROCESS_MEMORY_COUNTERS* p, unsigned long n)
{
    (void)h; (void)n;
    p->WorkingSetSize = p->PeakWorkingSetSize = p->PagefileUsage = p->PeakPagefileUsage = 0;
    return 1;
}
#endif
