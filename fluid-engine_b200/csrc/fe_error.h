// fe_error.h — the library's thread-local last-error message (fe_last_error).
#pragma once

// printf-style; replaces the message returned by fe_last_error() on this
// host thread.  Internal (not exported).
void fe_set_error_message(const char* fmt, ...);
