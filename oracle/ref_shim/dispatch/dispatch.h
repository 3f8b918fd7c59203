// Test infrastructure (oracle): the few libdispatch (GCD) names the reference engine's memory-pressure
// and idle-trim monitors use (src/session/engine.cpp:100-137). On this host build no event source is
// created, so the monitors never fire; queues are inert tokens and dispatch_sync_f runs inline.
#pragma once
#include <cstdint>

typedef struct spkref_dispatch_object* dispatch_queue_t;
typedef struct spkref_dispatch_object* dispatch_source_t;
typedef const struct spkref_dispatch_type* dispatch_source_type_t;
typedef uint64_t dispatch_time_t;
typedef void (*dispatch_function_t)(void*);

#define DISPATCH_QUEUE_SERIAL nullptr
#define DISPATCH_SOURCE_TYPE_MEMORYPRESSURE ((dispatch_source_type_t)1)
#define DISPATCH_SOURCE_TYPE_TIMER ((dispatch_source_type_t)2)
#define DISPATCH_MEMORYPRESSURE_NORMAL 0x01ul
#define DISPATCH_MEMORYPRESSURE_WARN 0x02ul
#define DISPATCH_MEMORYPRESSURE_CRITICAL 0x04ul
#define DISPATCH_TIME_NOW 0ull
#define DISPATCH_TIME_FOREVER (~0ull)
#ifndef NSEC_PER_SEC
#define NSEC_PER_SEC 1000000000ull
#endif

inline dispatch_queue_t dispatch_queue_create(const char*, const void*) {
    static int token;
    return reinterpret_cast<dispatch_queue_t>(&token);
}
inline dispatch_source_t dispatch_source_create(dispatch_source_type_t, uintptr_t, unsigned long, dispatch_queue_t) {
    return nullptr;
}
inline void dispatch_set_context(void*, void*) {}
inline void dispatch_source_set_event_handler_f(dispatch_source_t, dispatch_function_t) {}
inline unsigned long dispatch_source_get_data(dispatch_source_t) { return 0; }
inline dispatch_time_t dispatch_time(dispatch_time_t when, int64_t delta) { return when + uint64_t(delta); }
inline void dispatch_source_set_timer(dispatch_source_t, dispatch_time_t, uint64_t, uint64_t) {}
inline void dispatch_resume(void*) {}
inline void dispatch_source_cancel(dispatch_source_t) {}
inline void dispatch_sync_f(dispatch_queue_t, void* ctx, dispatch_function_t f) { f(ctx); }
inline void dispatch_release(void*) {}
