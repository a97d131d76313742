// The reference includes "NeoHookean.h" (VBD.cpp:4, NeoHookean.cpp:1) but ships Neohookean.h; on a
// case-sensitive file system this forwarder resolves the include to the shipped header.
#pragma once
#include "Neohookean.h"
