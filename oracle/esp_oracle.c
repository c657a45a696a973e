/* Placeholder translation unit of the oracle's C restatement; the FP64
 * pipeline is added here (test infrastructure only). */
int esp_oracle_version(void) { return 1; }
