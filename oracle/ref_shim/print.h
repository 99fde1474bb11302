// Empty host stand-in for the Poplar print header (oracle shim, test infrastructure only).
#pragma once
#include <cstdio>
