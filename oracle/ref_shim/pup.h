/* pup.h stand-in: see charm_stub.h.  TEST INFRASTRUCTURE. */
#include "charm_stub.h"
