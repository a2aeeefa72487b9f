/* Shim of the rsys 0.14 base header: the subset of macros and types the
 * reference's atmosphere hot-path files use (TEST INFRASTRUCTURE ONLY; it
 * exists to compile those files unmodified for the parity pin). */
#ifndef REF_SHIM_RSYS_H
#define REF_SHIM_RSYS_H

#include <assert.h>
#include <float.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define COMPILER_GCC

#define EXPORT_SYM __attribute__((visibility("default")))
#define IMPORT_SYM
#define LOCAL_SYM __attribute__((visibility("hidden")))

#define INLINE inline
#define FINLINE inline __attribute__((always_inline))

#ifdef __cplusplus
  #define BEGIN_DECLS extern "C" {
  #define END_DECLS }
#else
  #define BEGIN_DECLS
  #define END_DECLS
#endif

#define FUNC_NAME __func__

#ifdef NDEBUG
  #define ASSERT(C) (void)0
#else
  #define ASSERT(C) assert(C)
#endif

/* Evaluate C and abort when it is false, in every build */
#define CHK(C) do { if(!(C)) { \
  fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #C); abort(); } } while(0)
#define FATAL(Msg) do { fprintf(stderr, "%s", Msg); abort(); } while(0)

#define BIT(N) (1 << (N))
#define FOR_EACH(Id, Start, End) for((Id) = (Start); (Id) < (End); ++(Id))
#define MMIN(A, B) ((A) < (B) ? (A) : (B))
#define MMAX(A, B) ((A) > (B) ? (A) : (B))
#define CONTAINER_OF(Ptr, Type, Member) ((Type*)((char*)(Ptr) - offsetof(Type, Member)))
#define SPLIT2(A) (A)[0], (A)[1]
#define SPLIT3(A) (A)[0], (A)[1], (A)[2]
#define COUNTER __COUNTER__
#define ALIGNOF(Type) __alignof__(Type)
#define STR__(X) #X
#define STR(X) STR__(X)
#define IS_POW2(N) ((N) && !((N) & ((N) - 1)))
#define IS_ALIGNED(Addr, Align) (((uintptr_t)(Addr) & ((Align) - 1)) == 0)

typedef int res_T;
#define RES_OK 0
#define RES_BAD_ARG 1
#define RES_MEM_ERR 2
#define RES_IO_ERR 3
#define RES_UNKNOWN_ERR 4
#define RES_BAD_OP 5
#define RES_EOF 6

#endif
