// Empty shim (TEST INFRASTRUCTURE ONLY): the excised reference code needs nothing from this header.
#pragma once
