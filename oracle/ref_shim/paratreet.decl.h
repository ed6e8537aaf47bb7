/* paratreet.decl.h stand-in (Charm++ generated header): nothing of it is
 * needed by the gravity visitor's arithmetic.  TEST INFRASTRUCTURE. */
#include "charm_stub.h"

#ifndef PT_SHIM_DECL_EXTRAS_
#define PT_SHIM_DECL_EXTRAS_
/* examples/EwaldData.h derives from the generated CBase_EwaldData and takes a
 * CkCallback; EwaldInit only calls contribute(cb) on them. */
struct CkCallback {};
struct CBase_EwaldData {
  template <class T>
  void contribute(const T&) {}
};
#endif
