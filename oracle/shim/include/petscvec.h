/* Serial stand-in header for the oracle build of the reference (test infrastructure only). */
#pragma once
#include "pgshim.h"
