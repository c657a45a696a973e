"""Oracle: CPU restatements of the reference's ESP path and an FP64 direct
Ewald sum. Test infrastructure only -- imported by tests/, the smoke check
and the benchmark's CPU-baseline leg, never by the product path."""
