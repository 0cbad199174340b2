/* Empty stand-in for the CUDA runtime header: the reference kernel sources
 * include it, but the host-C++ build of those sources needs nothing from it.
 * Test infrastructure only (oracle/_ref). */
#pragma once
