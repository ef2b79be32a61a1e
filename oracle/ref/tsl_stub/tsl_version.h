// Minimal stand-in for the Tiny Shading Language version header (oracle build only).
#pragma once
#define TSL_VERSION_MAJOR 0
#define TSL_VERSION_MINOR 0
#define TSL_VERSION_PATCH 0
