/* SPLATT header stand-in for building the reference AdaTM files (oracle/_ref). */
#include "splatt_shim.h"
