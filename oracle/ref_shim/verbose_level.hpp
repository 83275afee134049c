// Shim: the verbosity levels the reference's utility.h declares (Off, Basic,
// Min, Max in that order), shared by every shim that compares against them.
#pragma once
enum VerboseLevel { Off, Basic, Min, Max };
