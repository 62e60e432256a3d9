// Empty stand-in for a CUDA header in the CPU checker build of the
// reference (oracle/_ref); ref_prelude.h provides what is used.  TEST
// INFRASTRUCTURE ONLY.
#pragma once
