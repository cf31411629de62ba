// Headless stand-ins for the MFC / Win32 names that the reference's
// integral and SCF translation units touch (TRACE, AfxMessageBox,
// _countof, the psapi process-memory query used only by an unused
// diagnostic).  Written for the oracle build; nothing here computes.
#pragma once
#include <cmath>
#include <cstddef>
#include <string>
using std::isinf;
using std::isnan;
#define TRACE(...) ((void)0)
inline int AfxMessageBox(const wchar_t *) { return 0; }
inline int AfxMessageBox(const char *) { return 0; }
#ifndef _countof
#define _countof(a) (sizeof(a) / sizeof((a)[0]))
#endif
typedef unsigned long DWORD;
typedef void *HANDLE;
struct PROCESS_MEMORY_COUNTERS {
  size_t PeakWorkingSetSize, WorkingSetSize, PagefileUsage, PeakPagefileUsage;
};
#define PROCESS_QUERY_INFORMATION 0
#define PROCESS_VM_READ 0
#ifndef FALSE
#define FALSE 0
#endif
inline HANDLE GetCurrentProcess() { return nullptr; }
inline DWORD GetProcessId(HANDLE) { return 0; }
inline HANDLE OpenProcess(int, int, DWORD) { return nullptr; }
inline bool GetProcessMemoryInfo(HANDLE, PROCESS_MEMORY_COUNTERS *, size_t) { return false; }
inline void CloseHandle(HANDLE) {}
struct CString {
  explicit CString(const char *) {}
  operator const wchar_t *() const { return L""; }
};
