/* Minimal configuration header used to compile the reference's own stencil
 * kernel (src/grid/operate.c, operate_inc.c, include/vectors.h) outside its
 * autotools build, for the CPU oracle.  Written for this project. */
#ifndef ORACLE_REF_STUB_CONFIG_H
#define ORACLE_REF_STUB_CONFIG_H
#define FC_FUNC_(name, NAME) name##_
#define FC_FUNC(name, NAME) name##_
#define HAVE_VEC 1
#define HAVE_M256D 1
#define HAVE_FMA3 1
#endif
