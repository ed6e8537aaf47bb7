/* paratreet.decl.h stand-in (Charm++ generated header): nothing of it is
 * needed by the gravity visitor's arithmetic.  TEST INFRASTRUCTURE. */
#include "charm_stub.h"
