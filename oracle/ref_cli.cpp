// Test infrastructure, not product code: the reference solver's own command-
// line program, linked by oracle/ref.mk from the reference's sources (their
// main() is compiled under another name so the same objects also build the
// harness library).  bench.py's reference arm runs it headless on the host
// cores as the stock CPU path of the hot path.
int nimbus_reference_cli_main(int argc, char** argv);

int main(int argc, char** argv) { return nimbus_reference_cli_main(argc, argv); }
