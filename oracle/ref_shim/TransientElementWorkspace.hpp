// Shim: the transient element workspace header (nothing of it is used by the
// code compiled here).
#pragma once
