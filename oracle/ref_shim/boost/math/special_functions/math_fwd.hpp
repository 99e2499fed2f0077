// Test-infrastructure shim: included by Twisty/PathWeighters.h, nothing used.
#pragma once
