// Empty host stand-in for a Poplar header (oracle shim, test infrastructure only).
#pragma once
